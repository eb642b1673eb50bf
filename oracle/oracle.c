/*
 * CPU oracle for the CasPhy tree-building hot path -- TEST INFRASTRUCTURE.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py (cpu_baseline and
 * --impl reference legs) load this file's shared object; the product
 * library never does.  Each function restates one reference executable's
 * semantics (host loop + device kernel) in plain C, citing the reference
 * lines it follows.  Paths are relative to the CasPhy source tree.
 *
 * Arithmetic is reproduced exactly:
 *  - joinEdgeIndel accumulates binary16 (`half`) weights one site at a time in
 *    ascending site order (cu/joinEdgeIndel.cu:73-79); here each add is done
 *    in double (exact for two binary16 operands) and rounded once to
 *    binary16, round-to-nearest-even, which is what the device `add.f16`
 *    does.  Weights are converted from the float64 file with one RNE
 *    rounding (cu/joinEdgeIndel.cu:296-298).
 *  - joinEdgeBitReverse / radiusNeighbor accumulate binary32 weights over
 *    the query's set bits in ascending bit order
 *    (cu/joinEdgeBitReverse.cu:61-69, cu/radiusNeighbor.cu:33-41).
 *  - argmax ties: larger value wins, then the smaller node index; the
 *    reduction starts from (-1, 0) (cu/joinEdgeIndel.cu:110-121).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef uint32_t u32;
typedef uint16_t u16;
typedef uint64_t u64;

/* ------------------------------------------------------------------ */
/* binary16                                                             */
/* ------------------------------------------------------------------ */

uint16_t oracle_f64_to_f16(double x) {
    u64 u;
    memcpy(&u, &x, 8);
    u16 sign = (u16)((u >> 48) & 0x8000u);
    u64 ax = u & 0x7FFFFFFFFFFFFFFFull;
    if (ax >= 0x7FF0000000000000ull) {
        if (ax > 0x7FF0000000000000ull) return (u16)(sign | 0x7E00u); /* NaN */
        return (u16)(sign | 0x7C00u);                                   /* inf */
    }
    double a;
    memcpy(&a, &ax, 8);
    if (a >= 65520.0) return (u16)(sign | 0x7C00u);
    if (a < 6.103515625e-05) { /* below 2^-14: subnormal grid of 2^-24 */
        double r = nearbyint(a * 16777216.0);
        return (u16)(sign | (u16)r);
    }
    int e;
    (void)frexp(a, &e);                 /* a = f * 2^e, f in [0.5,1) */
    double r = nearbyint(ldexp(a, 11 - e)); /* in [1024, 2048] */
    int E = e - 1;
    if (r >= 2048.0) { r = 1024.0; E += 1; }
    if (E > 15) return (u16)(sign | 0x7C00u);
    return (u16)(sign | (u16)(((E + 15) << 10) | ((int)r - 1024)));
}

double oracle_f16_to_f64(uint16_t h) {
    int s = h >> 15, e = (h >> 10) & 31, m = h & 1023;
    double v;
    if (e == 0) v = ldexp((double)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = ldexp((double)(m + 1024), e - 25);
    return s ? -v : v;
}

uint16_t oracle_f16_add(uint16_t a, uint16_t b) {
    return oracle_f64_to_f16(oracle_f16_to_f64(a) + oracle_f16_to_f64(b));
}

#define H_NEG_ONE ((u16)0xBC00u)

/* Non-zero: always emulate the binary16 adds (tests compare both paths). */
int oracle_force_f16 = 0;

static int nthreads_or_default(int n) { return n > 0 ? n : 1; }

/* ------------------------------------------------------------------ */
/* Shared greedy-join bookkeeping (cu/joinEdgeIndel.cu:321-468,          */
/* cu/joinEdgeBitReverse.cu:356-505).  Values are compared as doubles.  */
/* ------------------------------------------------------------------ */

typedef struct {
    u32 ntip, nnode, nedge;
    u32 *node2cache; /* nnode, ntip = invalid */
    u32 *cache2node; /* ntip, nnode = dead */
    u32 *valid;      /* ascending cache indices */
    u32 nvalid;
    u32 *localMaxIdx;
    u32 *rawEdge;    /* nedge*2, join order */
} JoinBook;

static int book_init(JoinBook *b, u32 ntip) {
    b->ntip = ntip;
    b->nnode = 2 * ntip - 1;
    b->nedge = 2 * ntip - 2;
    b->node2cache = (u32 *)malloc(sizeof(u32) * b->nnode);
    b->cache2node = (u32 *)malloc(sizeof(u32) * ntip);
    b->valid = (u32 *)malloc(sizeof(u32) * ntip);
    b->localMaxIdx = (u32 *)calloc(ntip, sizeof(u32));
    b->rawEdge = (u32 *)malloc(sizeof(u32) * (b->nedge ? b->nedge : 1) * 2);
    if (!b->node2cache || !b->cache2node || !b->valid || !b->localMaxIdx || !b->rawEdge)
        return ORACLE_ENOMEM;
    for (u32 i = 0; i < b->nnode; i++) b->node2cache[i] = i < ntip ? i : ntip;
    for (u32 i = 0; i < ntip; i++) { b->cache2node[i] = i; b->valid[i] = i; }
    b->nvalid = ntip;
    return ORACLE_OK;
}

static void book_free(JoinBook *b) {
    free(b->node2cache); free(b->cache2node); free(b->valid);
    free(b->localMaxIdx); free(b->rawEdge);
}

/* Removal keeps ascending order (cu/joinEdgeIndel.cu:430-437). */
static void book_remove_valid(JoinBook *b, u32 c) {
    u32 p = 0;
    while (p < b->nvalid && b->valid[p] < c) p++;
    if (p < b->nvalid && b->valid[p] == c) {
        memmove(b->valid + p, b->valid + p + 1, sizeof(u32) * (b->nvalid - p - 1));
        b->nvalid--;
    }
}

/* (v, i) beats (bv, bi)?  cu/joinEdgeIndel.cu:117 */
static inline int better(double v, u32 i, double bv, u32 bi) {
    return v > bv || (v == bv && i < bi);
}

/*
 * Pre-order relabel and output (cu/joinEdgeIndel.cu:488-558).  The
 * reference looks up, for the node on top of the stack, the first not yet
 * consumed edge (lowest index) whose parent is that node; internal node v's
 * edges sit at 2(v-ntip) and 2(v-ntip)+1, so a per-node cursor is the same
 * walk.  rawState(r) is the child state recorded for raw edge r; the root
 * state is rawState(nedge).
 */
static int dfs_output(const JoinBook *b, const u32 *rawState, u32 rowlen,
                      u32 *edge_out, u32 *state_out) {
    const u32 ntip = b->ntip, nnode = b->nnode, nedge = b->nedge;
    u32 *relabel = (u32 *)malloc(sizeof(u32) * nnode);
    u32 *stack = (u32 *)malloc(sizeof(u32) * (nedge + 1));
    unsigned char *cursor = (unsigned char *)calloc(nnode, 1);
    if (!relabel || !stack || !cursor) { free(relabel); free(stack); free(cursor); return ORACLE_ENOMEM; }
    for (u32 i = 0; i < nnode; i++) relabel[i] = i < ntip ? i : nnode;
    memcpy(state_out, rawState + (size_t)nedge * rowlen, sizeof(u32) * rowlen);
    u32 nstate = 1, nout = 0, count = ntip;
    long sp = 0;
    stack[0] = nedge; /* root node id */
    while (sp >= 0) {
        u32 v = stack[sp];
        if (v < ntip || cursor[v] >= 2) { sp--; continue; }
        u32 ei = 2 * (v - ntip) + cursor[v];
        cursor[v]++;
        u32 p = b->rawEdge[2 * ei], c = b->rawEdge[2 * ei + 1];
        stack[++sp] = c;
        if (relabel[p] == nnode) relabel[p] = count++;
        u32 lp = relabel[p], lc;
        if (relabel[c] == nnode) {
            memcpy(state_out + (size_t)nstate * rowlen, rawState + (size_t)ei * rowlen, sizeof(u32) * rowlen);
            nstate++;
            relabel[c] = count++;
        }
        lc = relabel[c];
        edge_out[2 * nout] = lp;
        edge_out[2 * nout + 1] = lc;
        nout++;
    }
    free(relabel); free(stack); free(cursor);
    return nout == nedge ? ORACLE_OK : ORACLE_EINTERNAL;
}

/* ------------------------------------------------------------------ */
/* joinEdgeIndel  (cu/joinEdgeIndel.cu:67-85, 87-99, 244-558)           */
/* ------------------------------------------------------------------ */

typedef struct {
    u32 ncol;
    const u32 *cache; /* ntip x ncol */
    const u16 *w16;   /* nState x ncol */
    const u16 *wint;  /* integer weights when every partial sum is exact, else NULL */
} IndelCtx;

/* calculateSharedKernel (cu/joinEdgeIndel.cu:67-85) for one pair.  When all
 * binary16 weights are integers in [0, 2048] and no score can exceed 2048,
 * every binary16 partial sum is exact and an integer sum is the same value;
 * the binary16 emulation is kept for every other weight table. */
static u16 indel_score(const IndelCtx *k, u32 q, u32 c) {
    const u32 *a = k->cache + (size_t)q * k->ncol, *r = k->cache + (size_t)c * k->ncol;
    if (k->wint) {
        u32 s = 0;
        for (u32 i = 0; i < k->ncol; i++) {
            u32 t = a[i];
            if (t == r[i] && t > 1) s += k->wint[(size_t)(t - 2) * k->ncol + i];
        }
        return oracle_f64_to_f16((double)s);
    }
    u16 acc = 0;
    for (u32 i = 0; i < k->ncol; i++) {
        u32 t = a[i];
        if (t == r[i] && t > 1) acc = oracle_f16_add(acc, k->w16[(size_t)(t - 2) * k->ncol + i]);
    }
    return acc;
}

static u16 *exact_int_weights(const u16 *w16, u32 nState, u32 ncol) {
    double total = 0;
    for (u32 i = 0; i < ncol; i++) {
        double mx = 0;
        for (u32 s = 0; s < nState; s++) {
            double v = oracle_f16_to_f64(w16[(size_t)s * ncol + i]);
            if (!(v >= 0 && v <= 2048 && v == floor(v))) return NULL;
            if (v > mx) mx = v;
        }
        total += mx;
    }
    if (total > 2048) return NULL;
    u16 *wi = (u16 *)malloc(sizeof(u16) * ((size_t)nState * ncol + 1));
    if (!wi) return NULL;
    for (size_t j = 0; j < (size_t)nState * ncol; j++) wi[j] = (u16)oracle_f16_to_f64(w16[j]);
    return wi;
}

/* updateAncestralKernel (cu/joinEdgeIndel.cu:87-99). */
static void indel_merge(u32 *a, const u32 *b, u32 n) {
    for (u32 i = 0; i < n; i++) {
        u32 x = a[i], y = b[i];
        if (x == 0) a[i] = y;
        else if (y >= 1 && x != y) a[i] = 1;
    }
}

/* ------------------------------------------------------------------ */
/* Column-scan engine for the indel join (integer weights only).        */
/* The same loop as oracle_join_indel below, with the pair scores of one */
/* query against many rows taken from a site-major u16 copy of the cache */
/* rows: for each site the query has edited, one contiguous pass over    */
/* that site's codes adds the weight where they are equal.  Exact        */
/* integer sums (the condition exact_int_weights checks) make the values */
/* and comparisons those of the binary16 loop; values are held as int,   */
/* -1 standing for the reference's -1 (H_NEG_ONE).  This is an execution */
/* strategy of the oracle for large trees; oracle_join_indel's row-wise  */
/* scoring is the default, and the CPU tests check that both engines     */
/* write the same tree.                                                  */
/* ------------------------------------------------------------------ */

/* Non-zero: oracle_join_indel uses the column-scan engine whenever the
 * weights are exact integers (oracle_force_f16 off). */
int oracle_indel_colscan = 0;

#define CS_CHUNK 1024u  /* candidates per accumulator block */
#define CS_QB 64u       /* queries per block in the initial pass */

typedef struct { u32 site; u16 code, w; } CsSite;

typedef struct {
    u32 ntip, ncol, cap;  /* cap: columns of colT (live and dead rows) */
    u16 *colT;            /* ncol x cap site-major codes */
    u32 *pos2cache;       /* column -> cache row, ntip when dead */
    u32 *cache2pos;       /* cache row -> column */
    const u16 *wint;
} ColScan;

/* Edited sites of cache row q with a non-zero weight. */
static u32 cs_query_sites(const u32 *row, u32 ncol, const u16 *wint, CsSite *out) {
    u32 n = 0;
    for (u32 i = 0; i < ncol; i++) {
        const u32 t = row[i];
        if (t > 1) {
            const u16 w = wint[(size_t)(t - 2) * ncol + i];
            if (w) { out[n].site = i; out[n].code = (u16)t; out[n].w = w; n++; }
        }
    }
    return n;
}

/* score[p] for every column p of colT against the query's sites. */
static void cs_scan(const ColScan *S, const CsSite *qs, u32 nqs, u16 *score, int nthreads) {
    const u32 cap = S->cap, nchunk = (cap + CS_CHUNK - 1) / CS_CHUNK;
#pragma omp parallel for num_threads(nthreads) schedule(static)
    for (long k = 0; k < (long)nchunk; k++) {
        const u32 c0 = (u32)k * CS_CHUNK, n = cap - c0 < CS_CHUNK ? cap - c0 : CS_CHUNK;
        u16 acc[CS_CHUNK];
        memset(acc, 0, sizeof(acc));
        for (u32 s = 0; s < nqs; s++) {
            const u16 *col = S->colT + (size_t)qs[s].site * cap + c0;
            const u16 t = qs[s].code, w = qs[s].w;
            for (u32 c = 0; c < n; c++) acc[c] += (u16)(col[c] == t ? w : 0);
        }
        memcpy(score + c0, acc, sizeof(u16) * n);
    }
}

/* Site-major copy of the live cache rows, columns in ascending cache order. */
static int cs_compact(ColScan *S, const u32 *cache, const JoinBook *b) {
    const u32 cap = b->nvalid;
    u16 *colT = (u16 *)malloc(sizeof(u16) * (size_t)S->ncol * (cap ? cap : 1));
    if (!colT) return ORACLE_ENOMEM;
    for (u32 p = 0; p < cap; p++) {
        const u32 c = b->valid[p];
        const u32 *row = cache + (size_t)c * S->ncol;
        for (u32 i = 0; i < S->ncol; i++) colT[(size_t)i * cap + p] = (u16)row[i];
        S->pos2cache[p] = c;
        S->cache2pos[c] = p;
    }
    free(S->colT);
    S->colT = colT;
    S->cap = cap;
    return ORACLE_OK;
}

static void cs_store_row(ColScan *S, u32 c, const u32 *row) {
    const u32 p = S->cache2pos[c];
    for (u32 i = 0; i < S->ncol; i++) S->colT[(size_t)i * S->cap + p] = (u16)row[i];
}

/* Initial upper-triangle local maxima (cu/joinEdgeIndel.cu:355-369) in
 * blocks of CS_QB queries, each site's codes read once per block. */
static void cs_initial(const ColScan *S, const u32 *cache, int *localMax, u32 *localMaxIdx, int nthreads) {
    const u32 ntip = S->ntip, ncol = S->ncol, nblk = (ntip + CS_QB - 1) / CS_QB;
#pragma omp parallel num_threads(nthreads)
    {
        u16 *acc = (u16 *)malloc(sizeof(u16) * CS_QB * CS_CHUNK);
        u16 *qcode = (u16 *)malloc(sizeof(u16) * CS_QB * ncol);
        u16 *qw = (u16 *)malloc(sizeof(u16) * CS_QB * ncol);
        u32 *act = (u32 *)malloc(sizeof(u32) * CS_QB * ncol);  /* active queries, site by site */
        u32 *actOff = (u32 *)malloc(sizeof(u32) * (ncol + 1));
#pragma omp for schedule(dynamic, 1)
        for (long blk = 0; blk < (long)nblk; blk++) {
            const u32 i0 = (u32)blk * CS_QB, nq = ntip - i0 < CS_QB ? ntip - i0 : CS_QB;
            int bv[CS_QB];
            u32 bi[CS_QB];
            for (u32 q = 0; q < nq; q++) {
                bv[q] = -1; bi[q] = 0;
                const u32 *row = cache + (size_t)(i0 + q) * ncol;
                for (u32 i = 0; i < ncol; i++) {
                    const u32 t = row[i];
                    const u16 w = t > 1 ? S->wint[(size_t)(t - 2) * ncol + i] : 0;
                    qcode[(size_t)i * CS_QB + q] = (u16)t;
                    qw[(size_t)i * CS_QB + q] = w;
                }
            }
            u32 na = 0;
            for (u32 i = 0; i < ncol; i++) {
                actOff[i] = na;
                for (u32 q = 0; q < nq; q++)
                    if (qw[(size_t)i * CS_QB + q]) act[na++] = q;
            }
            actOff[ncol] = na;
            for (u32 c0 = i0 + 1; c0 < ntip; c0 += CS_CHUNK) {
                const u32 n = ntip - c0 < CS_CHUNK ? ntip - c0 : CS_CHUNK;
                memset(acc, 0, sizeof(u16) * CS_QB * CS_CHUNK);
                for (u32 i = 0; i < ncol; i++) {
                    const u16 *col = S->colT + (size_t)i * S->cap + c0;
                    for (u32 a = actOff[i]; a < actOff[i + 1]; a++) {
                        const u32 q = act[a];
                        const u16 t = qcode[(size_t)i * CS_QB + q], w = qw[(size_t)i * CS_QB + q];
                        u16 *ac = acc + (size_t)q * CS_CHUNK;
                        for (u32 c = 0; c < n; c++) ac[c] += (u16)(col[c] == t ? w : 0);
                    }
                }
                /* ascending candidates, strict '>' keeps the smallest index */
                for (u32 q = 0; q < nq; q++) {
                    const u32 i = i0 + q;
                    const u16 *ac = acc + (size_t)q * CS_CHUNK;
                    for (u32 c = 0; c < n; c++) {
                        const u32 j = c0 + c;
                        if (j > i && (int)ac[c] > bv[q]) { bv[q] = ac[c]; bi[q] = j; }
                    }
                }
            }
            for (u32 q = 0; q < nq; q++) { localMax[i0 + q] = bv[q]; localMaxIdx[i0 + q] = bi[q]; }
        }
        free(acc); free(qcode); free(qw); free(act); free(actOff);
    }
    localMax[ntip - 1] = -1;
}

static int join_indel_colscan(u32 ntip, u32 ncol, u32 *cache, const u16 *wint, u32 *nodeSize, u32 minSize,
                              float minRatio, JoinBook *b, u32 *rawState, u64 *counts, int nthreads) {
    ColScan S;
    memset(&S, 0, sizeof(S));
    S.ntip = ntip; S.ncol = ncol; S.wint = wint;
    S.pos2cache = (u32 *)malloc(sizeof(u32) * ntip);
    S.cache2pos = (u32 *)malloc(sizeof(u32) * ntip);
    int *localMax = (int *)malloc(sizeof(int) * ntip);
    u16 *score = (u16 *)malloc(sizeof(u16) * ntip);
    CsSite *qs = (CsSite *)malloc(sizeof(CsSite) * ncol);
    int st = ORACLE_OK;
    u64 nStale = 0, nPairs = 0, nJoin = 0;
    if (!S.pos2cache || !S.cache2pos || !localMax || !score || !qs) { st = ORACLE_ENOMEM; goto out; }
    if ((st = cs_compact(&S, cache, b))) goto out;
    cs_initial(&S, cache, localMax, b->localMaxIdx, nthreads);
    nPairs = (u64)ntip * (ntip - 1) / 2;

    for (u32 nodeCount = ntip; nodeCount < b->nnode; nodeCount++) {
        u32 j1, j2, c1, c2;
        for (;;) {
            /* decision: best (value, smallest node) over the live rows (a
             * dead row holds (-1, nnode) and never wins) */
            int bv = -1;
            u32 bi = 0;
            for (u32 p = 0; p < b->nvalid; p++) {
                const u32 c = b->valid[p];
                const int v = localMax[c];
                const u32 node = b->cache2node[c];
                if (v > bv || (v == bv && node < bi)) { bv = v; bi = node; }
            }
            j1 = bi;
            if (j1 >= b->nnode) { st = ORACLE_EINTERNAL; goto out; }
            c1 = b->node2cache[j1];
            if (c1 >= ntip) { st = ORACLE_EINTERNAL; goto out; }
            j2 = b->localMaxIdx[c1];
            c2 = j2 < b->nnode ? b->node2cache[j2] : ntip;
            if (c2 < ntip) break;
            /* stale partner: rescore c1 against every valid row (:387-399) */
            nStale++;
            const u32 nqs = cs_query_sites(cache + (size_t)c1 * ncol, ncol, wint, qs);
            cs_scan(&S, qs, nqs, score, nthreads);
            nPairs += b->nvalid - 1;
            bv = -1; bi = 0;
            for (u32 p = 0; p < b->nvalid; p++) {
                const u32 c = b->valid[p];
                const int v = c == c1 ? -1 : (int)score[S.cache2pos[c]];
                const u32 node = b->cache2node[c];
                if (v > bv || (v == bv && node < bi)) { bv = v; bi = node; }
            }
            localMax[c1] = bv;
            b->localMaxIdx[c1] = bi;
        }
        const u32 r = nodeCount - ntip;
        u32 *row1 = cache + (size_t)c1 * ncol, *row2 = cache + (size_t)c2 * ncol;
        memcpy(rawState + (size_t)(2 * r) * ncol, row1, sizeof(u32) * ncol);
        memcpy(rawState + (size_t)(2 * r + 1) * ncol, row2, sizeof(u32) * ncol);
        const u32 s1 = nodeSize[j1], s2 = nodeSize[j2];
        if (s1 < minSize && (float)s1 * minRatio < (float)s2) memcpy(row1, row2, sizeof(u32) * ncol);
        else if (s2 < minSize && (float)s2 * minRatio < (float)s1) ;
        else indel_merge(row1, row2, ncol);
        nodeSize[nodeCount] = s1 + s2;
        b->rawEdge[4 * r] = nodeCount; b->rawEdge[4 * r + 1] = j1;
        b->rawEdge[4 * r + 2] = nodeCount; b->rawEdge[4 * r + 3] = j2;
        b->node2cache[j1] = ntip; b->node2cache[j2] = ntip; b->node2cache[nodeCount] = c1;
        b->cache2node[c1] = nodeCount; b->cache2node[c2] = b->nnode;
        book_remove_valid(b, c2);
        S.pos2cache[S.cache2pos[c2]] = ntip;
        if (b->nvalid * 2 < S.cap && S.cap > 4 * CS_CHUNK) {
            if ((st = cs_compact(&S, cache, b))) goto out;
        } else {
            cs_store_row(&S, c1, row1);
        }
        /* new node against every valid row, strict improvement (:439-463) */
        const u32 nqs = cs_query_sites(row1, ncol, wint, qs);
        cs_scan(&S, qs, nqs, score, nthreads);
        nPairs += b->nvalid - 1;
        for (u32 p = 0; p < b->nvalid; p++) {
            const u32 c = b->valid[p];
            if (c == c1) continue;
            const int v = score[S.cache2pos[c]];
            if (v > localMax[c]) { localMax[c] = v; b->localMaxIdx[c] = nodeCount; }
        }
        localMax[c1] = -1;
        localMax[c2] = -1;
        nJoin++;
    }
    memcpy(rawState + (size_t)(b->nnode - 1) * ncol, cache + (size_t)b->node2cache[b->nnode - 1] * ncol,
           sizeof(u32) * ncol);
out:
    counts[0] = nStale; counts[1] = nPairs; counts[2] = nJoin;
    free(S.colT); free(S.pos2cache); free(S.cache2pos); free(localMax); free(score); free(qs);
    return st;
}

int oracle_join_indel(uint32_t ntip, uint32_t ncol, const uint32_t *codes,
                      uint32_t nState, const double *w, const uint32_t *tipSize,
                      uint32_t minSize, float minRatio, uint32_t *edge_out,
                      uint32_t *state_out, uint64_t *stats, int nthreads) {
    if (ntip == 0 || ncol == 0) return ORACLE_EINVAL;
    nthreads = nthreads_or_default(nthreads);
    for (size_t i = 0; i < (size_t)ntip * ncol; i++)
        if (codes[i] > 1 && codes[i] - 2 >= nState) return ORACLE_ERANGE;
    const size_t nw = (size_t)nState * ncol;
    u16 *w16 = (u16 *)malloc(sizeof(u16) * (nw ? nw : 1));
    u32 *cache = (u32 *)malloc(sizeof(u32) * (size_t)ntip * ncol);
    u16 *localMax = (u16 *)malloc(sizeof(u16) * ntip);
    u16 *shared = (u16 *)malloc(sizeof(u16) * ntip);
    u32 nnode = 2 * ntip - 1;
    u32 *rawState = (u32 *)malloc(sizeof(u32) * (size_t)nnode * ncol);
    u32 *nodeSize = (u32 *)malloc(sizeof(u32) * (size_t)ntip * 2);
    u16 *wint = NULL;
    JoinBook b;
    int st = book_init(&b, ntip);
    if (st || !w16 || !cache || !localMax || !shared || !rawState || !nodeSize) { st = ORACLE_ENOMEM; goto done; }
    for (size_t i = 0; i < nw; i++) w16[i] = oracle_f64_to_f16(w[i]);
    memcpy(cache, codes, sizeof(u32) * (size_t)ntip * ncol);
    memcpy(nodeSize, tipSize, sizeof(u32) * ntip);
    wint = oracle_force_f16 ? NULL : exact_int_weights(w16, nState, ncol);
    IndelCtx k = {ncol, cache, w16, wint};
    u64 nStale = 0, nPairs = 0, nJoin = 0;
    if (wint && oracle_indel_colscan && nState + 1 <= 0xFFFFu) {
        u64 cnt[3];
        st = join_indel_colscan(ntip, ncol, cache, wint, nodeSize, minSize, minRatio, &b, rawState, cnt, nthreads);
        if (!st) st = dfs_output(&b, rawState, ncol, edge_out, state_out);
        if (!st && stats) { stats[0] = cnt[0]; stats[1] = cnt[1]; stats[2] = cnt[2]; }
        goto done;
    }

    /* initial upper-triangle local maxima (cu/joinEdgeIndel.cu:355-369) */
    for (u32 i = 0; i + 1 < ntip; i++) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long j = (long)i + 1; j < (long)ntip; j++) shared[j] = indel_score(&k, i, (u32)j);
        double bv = -1.0;
        u32 bi = 0;
        for (u32 j = i + 1; j < ntip; j++) {
            double v = oracle_f16_to_f64(shared[j]);
            if (better(v, j, bv, bi)) { bv = v; bi = j; }
        }
        localMax[i] = oracle_f64_to_f16(bv);
        b.localMaxIdx[i] = bi;
        nPairs += ntip - i - 1;
    }
    localMax[ntip - 1] = H_NEG_ONE;

    u32 nodeCount = ntip;
    while (nodeCount < b.nnode) {
        u32 j1, j2, c1, c2;
        for (;;) {
            double bv = -1.0;
            u32 bi = 0;
            for (u32 c = 0; c < ntip; c++) {
                double v = oracle_f16_to_f64(localMax[c]);
                if (better(v, b.cache2node[c], bv, bi)) { bv = v; bi = b.cache2node[c]; }
            }
            j1 = bi;
            if (j1 >= b.nnode) { st = ORACLE_EINTERNAL; goto done; }
            c1 = b.node2cache[j1];
            if (c1 >= ntip) { st = ORACLE_EINTERNAL; goto done; }
            j2 = b.localMaxIdx[c1];
            c2 = j2 < b.nnode ? b.node2cache[j2] : ntip;
            if (c2 < ntip) break;
            /* stale partner: rescore c1 against every valid row (:387-399) */
            nStale++;
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long p = 0; p < (long)b.nvalid; p++) {
                u32 c = b.valid[p];
                shared[c] = c == c1 ? H_NEG_ONE : indel_score(&k, c1, c);
            }
            nPairs += b.nvalid - 1;
            bv = -1.0;
            bi = 0;
            for (u32 p = 0; p < b.nvalid; p++) {
                u32 c = b.valid[p];
                double v = oracle_f16_to_f64(shared[c]);
                if (better(v, b.cache2node[c], bv, bi)) { bv = v; bi = b.cache2node[c]; }
            }
            localMax[c1] = oracle_f64_to_f16(bv);
            b.localMaxIdx[c1] = bi;
        }
        const u32 r = nodeCount - ntip;
        memcpy(rawState + (size_t)(2 * r) * ncol, cache + (size_t)c1 * ncol, sizeof(u32) * ncol);
        memcpy(rawState + (size_t)(2 * r + 1) * ncol, cache + (size_t)c2 * ncol, sizeof(u32) * ncol);
        u32 s1 = nodeSize[j1], s2 = nodeSize[j2];
        if (s1 < minSize && (float)s1 * minRatio < (float)s2) {
            memcpy(cache + (size_t)c1 * ncol, cache + (size_t)c2 * ncol, sizeof(u32) * ncol);
        } else if (s2 < minSize && (float)s2 * minRatio < (float)s1) {
            ;
        } else {
            indel_merge(cache + (size_t)c1 * ncol, cache + (size_t)c2 * ncol, ncol);
        }
        nodeSize[nodeCount] = s1 + s2;
        b.rawEdge[4 * r] = nodeCount; b.rawEdge[4 * r + 1] = j1;
        b.rawEdge[4 * r + 2] = nodeCount; b.rawEdge[4 * r + 3] = j2;
        b.node2cache[j1] = ntip; b.node2cache[j2] = ntip; b.node2cache[nodeCount] = c1;
        b.cache2node[c1] = nodeCount; b.cache2node[c2] = b.nnode;
        book_remove_valid(&b, c2);
        /* new node against every valid row, strict improvement (:439-463) */
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long p = 0; p < (long)b.nvalid; p++) {
            u32 c = b.valid[p];
            if (c != c1) shared[c] = indel_score(&k, c1, c);
        }
        nPairs += b.nvalid - 1;
        for (u32 p = 0; p < b.nvalid; p++) {
            u32 c = b.valid[p];
            if (c == c1) continue;
            if (oracle_f16_to_f64(shared[c]) > oracle_f16_to_f64(localMax[c])) {
                localMax[c] = shared[c];
                b.localMaxIdx[c] = nodeCount;
            }
        }
        localMax[c1] = H_NEG_ONE;
        localMax[c2] = H_NEG_ONE;
        nodeCount++;
        nJoin++;
    }
    memcpy(rawState + (size_t)(b.nnode - 1) * ncol, cache + (size_t)b.node2cache[nodeCount - 1] * ncol,
           sizeof(u32) * ncol);
    st = dfs_output(&b, rawState, ncol, edge_out, state_out);
    if (stats) { stats[0] = nStale; stats[1] = nPairs; stats[2] = nJoin; }
done:
    book_free(&b);
    free(w16); free(wint); free(cache); free(localMax); free(shared); free(rawState); free(nodeSize);
    return st;
}

/* ------------------------------------------------------------------ */
/* The greedy join on a phased schedule: fewer decision rounds, the same */
/* tree.  This is test infrastructure for a parallel engine (one phase = */
/* one round of decisions between grid barriers), not a restatement of   */
/* the reference; it checks two rules against the sequential joins above */
/* and below, for either scoring model.                                  */
/*  - Stale rescans run early: a row whose partner died is rescanned     */
/*    together with every other such row whose stored value beats the    */
/*    best fresh record (up to maxBatch rows, in decision order).  A     */
/*    rescan gives the row's true best over the live rows, and the join  */
/*    decision is the best true value, so rescanning early never changes */
/*    a decision.                                                        */
/*  - Two joins in one phase: when the phase joins a and b into n, let    */
/*    (c -> d) be the best record among the other rows.  If d is alive   */
/*    and is neither a nor b, and no row that n improves gets a record   */
/*    that beats (c -> d), the sequential loop's next decision is the    */
/*    join of c and d, so it is done in the same phase.                  */
/* Values are held as doubles: each model's stored values (binary16 or   */
/* binary32) convert exactly, so comparisons are those of its own loop.  */
/* ------------------------------------------------------------------ */

typedef struct {
    void *ctx;
    double (*score)(void *ctx, u32 q, u32 c);                  /* as the model stores it */
    void (*row_out)(void *ctx, u32 c, u32 *dst);               /* a cache row's output state */
    void (*merge)(void *ctx, u32 c1, u32 c2, u32 j1, u32 j2, u32 newNode); /* new node into row c1 */
    u32 rowlen;
} PhasedModel;

typedef struct {
    JoinBook b;
    const PhasedModel *m;
    u32 ntip, nodeCount;
    double *localMax, *shared;
    u32 *rawState;
    u64 nPairs;
    int nthreads;
} PhasedRun;

/* One join of cache rows c1 (node j1) and c2 (node j2), as the sequential
 * loops do it.  When `ok` is given it is cleared if a row improved by the
 * new node gets a record that beats (vcd, cNode). */
static void phased_join(PhasedRun *R, u32 j1, u32 j2, u32 c1, u32 c2, double vcd, u32 cNode, int *ok) {
    JoinBook *b = &R->b;
    const PhasedModel *m = R->m;
    const u32 ntip = R->ntip, nodeCount = R->nodeCount, r = nodeCount - ntip;
    m->row_out(m->ctx, c1, R->rawState + (size_t)(2 * r) * m->rowlen);
    m->row_out(m->ctx, c2, R->rawState + (size_t)(2 * r + 1) * m->rowlen);
    m->merge(m->ctx, c1, c2, j1, j2, nodeCount);
    b->rawEdge[4 * r] = nodeCount; b->rawEdge[4 * r + 1] = j1;
    b->rawEdge[4 * r + 2] = nodeCount; b->rawEdge[4 * r + 3] = j2;
    b->node2cache[j1] = ntip; b->node2cache[j2] = ntip; b->node2cache[nodeCount] = c1;
    b->cache2node[c1] = nodeCount; b->cache2node[c2] = b->nnode;
    book_remove_valid(b, c2);
    double *shared = R->shared;
#pragma omp parallel for num_threads(R->nthreads) schedule(static)
    for (long p = 0; p < (long)b->nvalid; p++) {
        u32 c = b->valid[p];
        if (c != c1) shared[c] = m->score(m->ctx, c1, c);
    }
    R->nPairs += b->nvalid - 1;
    for (u32 p = 0; p < b->nvalid; p++) {
        u32 c = b->valid[p];
        if (c == c1) continue;
        if (shared[c] > R->localMax[c]) {
            if (ok && better(shared[c], b->cache2node[c], vcd, cNode)) *ok = 0;
            R->localMax[c] = shared[c];
            b->localMaxIdx[c] = nodeCount;
        }
    }
    R->localMax[c1] = -1.0;
    R->localMax[c2] = -1.0;
    R->nodeCount++;
}

/* Rescan of cache row t against every valid row (the stale step). */
static void phased_rescan(PhasedRun *R, u32 t) {
    JoinBook *b = &R->b;
    const PhasedModel *m = R->m;
    double *shared = R->shared;
#pragma omp parallel for num_threads(R->nthreads) schedule(static)
    for (long p = 0; p < (long)b->nvalid; p++) {
        u32 c = b->valid[p];
        shared[c] = c == t ? -1.0 : m->score(m->ctx, t, c);
    }
    R->nPairs += b->nvalid - 1;
    double bv = -1.0;
    u32 bi = 0;
    for (u32 p = 0; p < b->nvalid; p++) {
        u32 c = b->valid[p];
        if (better(shared[c], b->cache2node[c], bv, bi)) { bv = shared[c]; bi = b->cache2node[c]; }
    }
    R->localMax[t] = bv;
    b->localMaxIdx[t] = bi;
}

static int phased_fresh(const PhasedRun *R, u32 c) {
    const u32 d = R->b.localMaxIdx[c];
    return d < R->b.nnode && R->b.node2cache[d] < R->ntip;
}

/* stats (nullable): [0] stale rescans, [1] pair-scores, [2] joins, [3]
 * phases, [4] phases with two joins, [5] pairs given up because a table of
 * each CTA's top two records could not vouch for them.
 * tableCTAs > 0 models such a table: the live rows are split by rank into
 * tableCTAs equal ranges (as if renumbered densely every phase), and a
 * pair is given up when a and b are the two best records of one range
 * that holds more live records, which hides that range's third best. */

/* Position of cache row c among the valid rows (ascending). */
static u32 valid_rank(const JoinBook *b, u32 c) {
    u32 lo = 0, hi = b->nvalid;
    while (lo < hi) {
        const u32 mid = (lo + hi) / 2;
        if (b->valid[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* Would a top-2-per-range table hide the best record outside rows c1, c2? */
static int table_hides(const PhasedRun *R, u32 c1, u32 c2, u32 tableCTAs) {
    const JoinBook *b = &R->b;
    const u32 per = (b->nvalid + tableCTAs - 1) / tableCTAs;
    const u32 t = valid_rank(b, c1) / per;
    if (valid_rank(b, c2) / per != t) return 0;
    const u32 p0 = t * per, p1 = p0 + per < b->nvalid ? p0 + per : b->nvalid;
    double v0 = -1.0, v1 = -1.0;
    u32 n0 = 0, n1 = 0, s0 = ~0u, s1 = ~0u, cnt = 0;
    for (u32 p = p0; p < p1; p++) {
        const u32 c = b->valid[p];
        const double v = R->localMax[c];
        if (v < 0) continue;
        cnt++;
        const u32 node = b->cache2node[c];
        if (better(v, node, v0, n0)) { v1 = v0; n1 = n0; s1 = s0; v0 = v; n0 = node; s0 = c; }
        else if (better(v, node, v1, n1)) { v1 = v; n1 = node; s1 = c; }
    }
    return cnt > 2 && ((s0 == c1 && s1 == c2) || (s0 == c2 && s1 == c1));
}

static int phased_join_run(const PhasedModel *m, u32 ntip, u32 maxBatch, int pairJoins, u32 tableCTAs, u32 *edge_out,
                           u32 *state_out, u64 *stats, int nthreads) {
    if (ntip == 0 || maxBatch == 0) return ORACLE_EINVAL;
    PhasedRun R;
    memset(&R, 0, sizeof(R));
    R.m = m;
    R.ntip = ntip;
    R.nthreads = nthreads_or_default(nthreads);
    const u32 nnode = 2 * ntip - 1;
    u32 *batch = (u32 *)malloc(sizeof(u32) * ntip);
    R.localMax = (double *)malloc(sizeof(double) * ntip);
    R.shared = (double *)malloc(sizeof(double) * ntip);
    R.rawState = (u32 *)malloc(sizeof(u32) * (size_t)nnode * m->rowlen);
    int st = book_init(&R.b, ntip);
    if (st || !batch || !R.localMax || !R.shared || !R.rawState) { st = ORACLE_ENOMEM; goto done; }
    JoinBook *b = &R.b;
    u64 nStale = 0, nJoin = 0, nPhase = 0, nPaired = 0, nHidden = 0, nRiding = 0;

    for (u32 i = 0; i + 1 < ntip; i++) {
#pragma omp parallel for num_threads(R.nthreads) schedule(static)
        for (long j = (long)i + 1; j < (long)ntip; j++) R.shared[j] = m->score(m->ctx, i, (u32)j);
        double bv = -1.0;
        u32 bi = 0;
        for (u32 j = i + 1; j < ntip; j++)
            if (better(R.shared[j], j, bv, bi)) { bv = R.shared[j]; bi = j; }
        R.localMax[i] = bv;
        b->localMaxIdx[i] = bi;
        R.nPairs += ntip - i - 1;
    }
    R.localMax[ntip - 1] = -1.0;
    R.nodeCount = ntip;

    while (R.nodeCount < nnode) {
        double bv = -1.0, fv = -1.0;
        u32 bi = 0, fi = 0;
        for (u32 c = 0; c < ntip; c++) {
            const double v = R.localMax[c];
            const u32 node = b->cache2node[c];
            if (better(v, node, bv, bi)) { bv = v; bi = node; }
            if (node < nnode && phased_fresh(&R, c) && better(v, node, fv, fi)) { fv = v; fi = node; }
        }
        u32 j1 = bi;
        if (j1 >= nnode || b->node2cache[j1] >= ntip) { st = ORACLE_EINTERNAL; goto done; }
        u32 jj = j1;
        if (!phased_fresh(&R, b->node2cache[j1])) {
            const u32 c1 = b->node2cache[j1];
            /* one phase: the stale rows that beat the best fresh record, best first */
            u32 n = 0;
            for (u32 c = 0; c < ntip; c++) {
                const u32 node = b->cache2node[c];
                if (node >= nnode || phased_fresh(&R, c)) continue;
                if (R.localMax[c] >= 0 && better(R.localMax[c], node, fv, fi)) batch[n++] = c;
            }
            for (u32 x = 1; x < n; x++) { /* insertion sort, decision order */
                const u32 t = batch[x];
                u32 y = x;
                while (y > 0 && better(R.localMax[t], b->cache2node[t], R.localMax[batch[y - 1]],
                                       b->cache2node[batch[y - 1]])) {
                    batch[y] = batch[y - 1];
                    y--;
                }
                batch[y] = t;
            }
            if (n == 0 || batch[0] != c1) { st = ORACLE_EINTERNAL; goto done; }
            if (n > maxBatch) n = maxBatch;
            for (u32 x = 0; x < n; x++) phased_rescan(&R, batch[x]);
            nStale += n;
            nPhase++;
            /* the join of the best fresh record rides along when it is still
             * the decision after the rescans (bit 1 of pairJoins) */
            if (!(pairJoins & 2) || fv < 0) continue;
            double b2 = -1.0;
            u32 i2 = 0;
            for (u32 c = 0; c < ntip; c++)
                if (better(R.localMax[c], b->cache2node[c], b2, i2)) { b2 = R.localMax[c]; i2 = b->cache2node[c]; }
            if (i2 != fi || !phased_fresh(&R, b->node2cache[fi])) continue;
            jj = fi;
            nRiding++;
        } else {
            nPhase++;
        }
        const u32 c1 = b->node2cache[jj];
        j1 = jj;
        const u32 j2 = b->localMaxIdx[c1], c2 = b->node2cache[j2];
        /* the best record among the other rows, before this join */
        double vcd = -1.0;
        u32 cNode = 0;
        for (u32 c = 0; c < ntip; c++) {
            if (c == c1 || c == c2) continue;
            if (better(R.localMax[c], b->cache2node[c], vcd, cNode)) { vcd = R.localMax[c]; cNode = b->cache2node[c]; }
        }
        int ok = 0;
        u32 cc = ntip, dNode = nnode;
        if ((pairJoins & 1) && vcd >= 0 && cNode < nnode && b->node2cache[cNode] < ntip) {
            cc = b->node2cache[cNode];
            dNode = b->localMaxIdx[cc];
            ok = phased_fresh(&R, cc) && dNode != j1 && dNode != j2;
            if (ok && tableCTAs && table_hides(&R, c1, c2, tableCTAs)) {
                ok = 0;
                nHidden++;
            }
        }
        phased_join(&R, j1, j2, c1, c2, vcd, cNode, ok ? &ok : NULL);
        nJoin++;
        if (ok && R.nodeCount < nnode) {
            phased_join(&R, cNode, dNode, cc, b->node2cache[dNode], 0.0, 0, NULL);
            nJoin++;
            nPaired++;
        }
    }
    m->row_out(m->ctx, b->node2cache[R.nodeCount - 1], R.rawState + (size_t)(nnode - 1) * m->rowlen);
    st = dfs_output(b, R.rawState, m->rowlen, edge_out, state_out);
    if (stats) {
        stats[0] = nStale; stats[1] = R.nPairs; stats[2] = nJoin; stats[3] = nPhase; stats[4] = nPaired;
        stats[5] = nHidden; stats[6] = nRiding;
    }
done:
    book_free(&R.b);
    free(batch); free(R.localMax); free(R.shared); free(R.rawState);
    return st;
}

/* Indel model for the phased join (the same steps as oracle_join_indel). */
typedef struct {
    IndelCtx k;
    u32 *cache, *nodeSize;
    u32 ncol, minSize;
    float minRatio;
} IndelPhased;

static double ip_score(void *p, u32 q, u32 c) {
    return oracle_f16_to_f64(indel_score(&((IndelPhased *)p)->k, q, c));
}

static void ip_row(void *p, u32 c, u32 *dst) {
    IndelPhased *x = (IndelPhased *)p;
    memcpy(dst, x->cache + (size_t)c * x->ncol, sizeof(u32) * x->ncol);
}

static void ip_merge(void *p, u32 c1, u32 c2, u32 j1, u32 j2, u32 newNode) {
    IndelPhased *x = (IndelPhased *)p;
    const u32 s1 = x->nodeSize[j1], s2 = x->nodeSize[j2], ncol = x->ncol;
    if (s1 < x->minSize && (float)s1 * x->minRatio < (float)s2)
        memcpy(x->cache + (size_t)c1 * ncol, x->cache + (size_t)c2 * ncol, sizeof(u32) * ncol);
    else if (!(s2 < x->minSize && (float)s2 * x->minRatio < (float)s1))
        indel_merge(x->cache + (size_t)c1 * ncol, x->cache + (size_t)c2 * ncol, ncol);
    x->nodeSize[newNode] = s1 + s2;
}

int oracle_join_indel_phased(uint32_t ntip, uint32_t ncol, const uint32_t *codes, uint32_t nState,
                             const double *w, const uint32_t *tipSize, uint32_t minSize, float minRatio,
                             uint32_t maxBatch, int pairJoins, uint32_t tableCTAs, uint32_t *edge_out,
                             uint32_t *state_out, uint64_t *stats, int nthreads) {
    if (ntip == 0 || ncol == 0 || maxBatch == 0) return ORACLE_EINVAL;
    for (size_t i = 0; i < (size_t)ntip * ncol; i++)
        if (codes[i] > 1 && codes[i] - 2 >= nState) return ORACLE_ERANGE;
    const size_t nw = (size_t)nState * ncol;
    IndelPhased x;
    memset(&x, 0, sizeof(x));
    u16 *w16 = (u16 *)malloc(sizeof(u16) * (nw ? nw : 1));
    x.cache = (u32 *)malloc(sizeof(u32) * (size_t)ntip * ncol);
    x.nodeSize = (u32 *)malloc(sizeof(u32) * (size_t)ntip * 2);
    int st = ORACLE_ENOMEM;
    if (w16 && x.cache && x.nodeSize) {
        for (size_t i = 0; i < nw; i++) w16[i] = oracle_f64_to_f16(w[i]);
        memcpy(x.cache, codes, sizeof(u32) * (size_t)ntip * ncol);
        memcpy(x.nodeSize, tipSize, sizeof(u32) * ntip);
        x.ncol = ncol; x.minSize = minSize; x.minRatio = minRatio;
        x.k.ncol = ncol; x.k.cache = x.cache; x.k.w16 = w16;
        x.k.wint = oracle_force_f16 ? NULL : exact_int_weights(w16, nState, ncol);
        PhasedModel m = {&x, ip_score, ip_row, ip_merge, ncol};
        st = phased_join_run(&m, ntip, maxBatch, pairJoins, tableCTAs, edge_out, state_out, stats, nthreads);
        free((void *)x.k.wint);
    }
    free(w16); free(x.cache); free(x.nodeSize);
    return st;
}

/* ------------------------------------------------------------------ */
/* joinEdgeBitReverse (cu/joinEdgeBitReverse.cu:53-121, 285-597)       */
/* ------------------------------------------------------------------ */

typedef struct {
    u32 nbin;
    const u32 *seq;
    const float *wf;
} BitCtx;

/* calculateSharedKernel: float sum over the query's set bits in ascending
 * order where the candidate bit is set (cu/joinEdgeBitReverse.cu:61-69,
 * bit list built by calculateSharedPacked :235-244). */
static float bit_score(const BitCtx *k, u32 q, u32 c) {
    const u32 *a = k->seq + (size_t)q * k->nbin, *r = k->seq + (size_t)c * k->nbin;
    float acc = 0.0f;
    for (u32 j = 0; j < k->nbin; j++) {
        u32 v = a[j] & r[j];
        while (v) {
            int bit = __builtin_ctz(v);
            acc += k->wf[j * 32 + bit];
            v &= v - 1;
        }
    }
    return acc;
}

int oracle_join_bit(uint32_t ntip, uint32_t nbin, const uint32_t *words,
                    const double *w, int ancestralType, uint32_t *edge_out,
                    uint32_t *state_out, uint64_t *stats, int nthreads) {
    if (ntip == 0 || nbin == 0) return ORACLE_EINVAL;
    nthreads = nthreads_or_default(nthreads);
    const u32 nsite = nbin * 32;
    float *wf = (float *)malloc(sizeof(float) * nsite);
    u32 *seq = (u32 *)malloc(sizeof(u32) * (size_t)ntip * nbin);
    u32 *bis = (u32 *)calloc((size_t)ntip * nbin, sizeof(u32));
    float *localMax = (float *)malloc(sizeof(float) * ntip);
    float *shared = (float *)malloc(sizeof(float) * ntip);
    u32 nnode = 2 * ntip - 1;
    u32 *rawState = (u32 *)malloc(sizeof(u32) * (size_t)nnode * nbin);
    JoinBook b;
    int st = book_init(&b, ntip);
    if (st || !wf || !seq || !bis || !localMax || !shared || !rawState) { st = ORACLE_ENOMEM; goto done; }
    for (u32 i = 0; i < nsite; i++) wf[i] = (float)w[i];
    memcpy(seq, words, sizeof(u32) * (size_t)ntip * nbin);
    BitCtx k = {nbin, seq, wf};
    u64 nStale = 0, nPairs = 0, nJoin = 0;

    for (u32 i = 0; i + 1 < ntip; i++) {
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long j = (long)i + 1; j < (long)ntip; j++) shared[j] = bit_score(&k, i, (u32)j);
        float bv = -1.0f;
        u32 bi = 0;
        for (u32 j = i + 1; j < ntip; j++)
            if (better(shared[j], j, bv, bi)) { bv = shared[j]; bi = j; }
        localMax[i] = bv;
        b.localMaxIdx[i] = bi;
        nPairs += ntip - i - 1;
    }
    localMax[ntip - 1] = -1.0f;

    u32 nodeCount = ntip;
    while (nodeCount < b.nnode) {
        u32 j1, j2, c1, c2;
        for (;;) {
            float bv = -1.0f;
            u32 bi = 0;
            for (u32 c = 0; c < ntip; c++)
                if (better(localMax[c], b.cache2node[c], bv, bi)) { bv = localMax[c]; bi = b.cache2node[c]; }
            j1 = bi;
            if (j1 >= b.nnode) { st = ORACLE_EINTERNAL; goto done; }
            c1 = b.node2cache[j1];
            if (c1 >= ntip) { st = ORACLE_EINTERNAL; goto done; }
            j2 = b.localMaxIdx[c1];
            c2 = j2 < b.nnode ? b.node2cache[j2] : ntip;
            if (c2 < ntip) break;
            nStale++;
#pragma omp parallel for num_threads(nthreads) schedule(static)
            for (long p = 0; p < (long)b.nvalid; p++) {
                u32 c = b.valid[p];
                shared[c] = c == c1 ? -1.0f : bit_score(&k, c1, c);
            }
            nPairs += b.nvalid - 1;
            bv = -1.0f;
            bi = 0;
            for (u32 p = 0; p < b.nvalid; p++) {
                u32 c = b.valid[p];
                if (better(shared[c], b.cache2node[c], bv, bi)) { bv = shared[c]; bi = b.cache2node[c]; }
            }
            localMax[c1] = bv;
            b.localMaxIdx[c1] = bi;
        }
        const u32 r = nodeCount - ntip;
        /* nodeStateOutputKernel: seq & ~bistate (:115-121, :436-443) */
        for (u32 j = 0; j < nbin; j++) {
            rawState[(size_t)(2 * r) * nbin + j] = seq[(size_t)c1 * nbin + j] & ~bis[(size_t)c1 * nbin + j];
            rawState[(size_t)(2 * r + 1) * nbin + j] = seq[(size_t)c2 * nbin + j] & ~bis[(size_t)c2 * nbin + j];
        }
        for (u32 j = 0; j < nbin; j++) {
            u32 s1 = seq[(size_t)c1 * nbin + j], s2 = seq[(size_t)c2 * nbin + j];
            u32 b1 = bis[(size_t)c1 * nbin + j], b2 = bis[(size_t)c2 * nbin + j];
            if (ancestralType == 0) { /* updateAncestralKernel (:77-95) */
                u32 diff = s1 ^ s2;
                u32 conflict = diff & (b1 | b2);
                seq[(size_t)c1 * nbin + j] = (s1 | s2) & ~conflict;
                bis[(size_t)c1 * nbin + j] = (diff & ~(b1 ^ b2)) | (b1 & b2);
            } else { /* updateAncestralKernel2 (:97-113) */
                seq[(size_t)c1 * nbin + j] = (s1 & s2) | (b1 & s2) | (b2 & s1);
                bis[(size_t)c1 * nbin + j] = (s1 ^ s2) & ~(b1 | b2);
            }
        }
        b.rawEdge[4 * r] = nodeCount; b.rawEdge[4 * r + 1] = j1;
        b.rawEdge[4 * r + 2] = nodeCount; b.rawEdge[4 * r + 3] = j2;
        b.node2cache[j1] = ntip; b.node2cache[j2] = ntip; b.node2cache[nodeCount] = c1;
        b.cache2node[c1] = nodeCount; b.cache2node[c2] = b.nnode;
        book_remove_valid(&b, c2);
#pragma omp parallel for num_threads(nthreads) schedule(static)
        for (long p = 0; p < (long)b.nvalid; p++) {
            u32 c = b.valid[p];
            if (c != c1) shared[c] = bit_score(&k, c1, c);
        }
        nPairs += b.nvalid - 1;
        for (u32 p = 0; p < b.nvalid; p++) {
            u32 c = b.valid[p];
            if (c == c1) continue;
            if (shared[c] > localMax[c]) { localMax[c] = shared[c]; b.localMaxIdx[c] = nodeCount; }
        }
        localMax[c1] = -1.0f;
        localMax[c2] = -1.0f;
        nodeCount++;
        nJoin++;
    }
    {
        u32 c = b.node2cache[nodeCount - 1];
        for (u32 j = 0; j < nbin; j++)
            rawState[(size_t)(b.nnode - 1) * nbin + j] = seq[(size_t)c * nbin + j] & ~bis[(size_t)c * nbin + j];
    }
    st = dfs_output(&b, rawState, nbin, edge_out, state_out);
    if (stats) { stats[0] = nStale; stats[1] = nPairs; stats[2] = nJoin; }
done:
    book_free(&b);
    free(wf); free(seq); free(bis); free(localMax); free(shared); free(rawState);
    return st;
}

/* Bit model for the phased join (the same steps as oracle_join_bit). */
typedef struct {
    BitCtx k;
    u32 *seq, *bis;
    u32 nbin;
    int ancestralType;
} BitPhased;

static double bp_score(void *p, u32 q, u32 c) { return (double)bit_score(&((BitPhased *)p)->k, q, c); }

static void bp_row(void *p, u32 c, u32 *dst) {
    BitPhased *x = (BitPhased *)p;
    for (u32 j = 0; j < x->nbin; j++) dst[j] = x->seq[(size_t)c * x->nbin + j] & ~x->bis[(size_t)c * x->nbin + j];
}

static void bp_merge(void *p, u32 c1, u32 c2, u32 j1, u32 j2, u32 newNode) {
    BitPhased *x = (BitPhased *)p;
    const u32 nbin = x->nbin;
    for (u32 j = 0; j < nbin; j++) {
        u32 s1 = x->seq[(size_t)c1 * nbin + j], s2 = x->seq[(size_t)c2 * nbin + j];
        u32 b1 = x->bis[(size_t)c1 * nbin + j], b2 = x->bis[(size_t)c2 * nbin + j];
        if (x->ancestralType == 0) {
            u32 diff = s1 ^ s2, conflict = diff & (b1 | b2);
            x->seq[(size_t)c1 * nbin + j] = (s1 | s2) & ~conflict;
            x->bis[(size_t)c1 * nbin + j] = (diff & ~(b1 ^ b2)) | (b1 & b2);
        } else {
            x->seq[(size_t)c1 * nbin + j] = (s1 & s2) | (b1 & s2) | (b2 & s1);
            x->bis[(size_t)c1 * nbin + j] = (s1 ^ s2) & ~(b1 | b2);
        }
    }
}

int oracle_join_bit_phased(uint32_t ntip, uint32_t nbin, const uint32_t *words, const double *w,
                           int ancestralType, uint32_t maxBatch, int pairJoins, uint32_t tableCTAs,
                           uint32_t *edge_out, uint32_t *state_out, uint64_t *stats, int nthreads) {
    if (ntip == 0 || nbin == 0 || maxBatch == 0) return ORACLE_EINVAL;
    const u32 nsite = nbin * 32;
    BitPhased x;
    memset(&x, 0, sizeof(x));
    float *wf = (float *)malloc(sizeof(float) * nsite);
    x.seq = (u32 *)malloc(sizeof(u32) * (size_t)ntip * nbin);
    x.bis = (u32 *)calloc((size_t)ntip * nbin, sizeof(u32));
    int st = ORACLE_ENOMEM;
    if (wf && x.seq && x.bis) {
        for (u32 i = 0; i < nsite; i++) wf[i] = (float)w[i];
        memcpy(x.seq, words, sizeof(u32) * (size_t)ntip * nbin);
        x.nbin = nbin;
        x.ancestralType = ancestralType ? 1 : 0;
        x.k.nbin = nbin; x.k.seq = x.seq; x.k.wf = wf;
        PhasedModel m = {&x, bp_score, bp_row, bp_merge, nbin};
        st = phased_join_run(&m, ntip, maxBatch, pairJoins, tableCTAs, edge_out, state_out, stats, nthreads);
    }
    free(wf); free(x.seq); free(x.bis);
    return st;
}

/* ------------------------------------------------------------------ */
/* nodeKeepIndel (cu/nodeKeepIndel.cu:32-48,130-152)                    */
/* nodeKeepBit   (cu/nodeKeepBit.cu:33-51,186-211)                      */
/* ------------------------------------------------------------------ */

static int node_keep_common(int bitmode, u32 nnodeRows, u32 ncol, const u32 *nodeState,
                            u32 nedge, const u32 *edge, u32 nRetain, const u32 *outmat,
                            u32 cutoff, u32 *out_nodes, u32 *nout) {
    const u32 ntip = nnodeRows + 1;
    u32 currentNode = ntip - 1, flag = 0, n = 0;
    for (u32 i = 0; i < nedge; i++) {
        u32 parent = edge[2 * i], child = edge[2 * i + 1];
        if (!(child + 1 > ntip)) continue;
        if (flag == 1 && currentNode <= parent) continue;
        u32 row = child - ntip;
        if (row >= nnodeRows) return ORACLE_ERANGE;
        const u32 *ref = nodeState + (size_t)row * ncol;
        flag = 1;
        for (u32 j = 0; j < nRetain && flag; j++) {
            const u32 *o = outmat + (size_t)j * ncol;
            u32 cnt = 0;
            if (bitmode) {
                for (u32 t = 0; t < ncol; t++) cnt += (u32)__builtin_popcount(ref[t] & ~o[t]);
            } else {
                for (u32 t = 0; t < ncol; t++)
                    if (ref[t] > 1 && o[t] != ref[t] && o[t] >= 1) cnt++;
            }
            if (cnt < cutoff) flag = 0;
        }
        if (flag == 1) { currentNode = child; out_nodes[n++] = child; }
    }
    *nout = n;
    return ORACLE_OK;
}

int oracle_node_keep_indel(uint32_t nnodeRows, uint32_t ncol, const uint32_t *nodeState,
                           uint32_t nedge, const uint32_t *edge, uint32_t nRetain,
                           const uint32_t *outmat, uint32_t cutoff,
                           uint32_t *out_nodes, uint32_t *nout) {
    return node_keep_common(0, nnodeRows, ncol, nodeState, nedge, edge, nRetain, outmat, cutoff, out_nodes, nout);
}

int oracle_node_keep_bit(uint32_t nnodeRows, uint32_t nbin, const uint32_t *nodeState,
                         uint32_t nedge, const uint32_t *edge, uint32_t nRetain,
                         const uint32_t *outmat, uint32_t cutoff,
                         uint32_t *out_nodes, uint32_t *nout) {
    return node_keep_common(1, nnodeRows, nbin, nodeState, nedge, edge, nRetain, outmat, cutoff, out_nodes, nout);
}

/* ------------------------------------------------------------------ */
/* radiusNeighbor (cu/radiusNeighbor.cu:26-50, 162-437).  The output of  */
/* the host mirror loop (:383-425) is, for every row i, the ascending   */
/* list {j : score(i,j) >= radius}; the score is symmetric because both */
/* directions add the same weights in the same ascending bit order.     */
/* ------------------------------------------------------------------ */

static float radius_bit_score(const u32 *bmat, u32 nrow, u32 ntip, const float *wf, u32 q, u32 c) {
    float acc = 0.0f;
    for (u32 j = 0; j < nrow; j++) {
        u32 v = bmat[(size_t)j * ntip + q] & bmat[(size_t)j * ntip + c];
        while (v) {
            int bit = __builtin_ctz(v);
            acc += wf[j * 32 + bit];
            v &= v - 1;
        }
    }
    return acc;
}

/* Emit lists from a predicate evaluated per (i,j). */
typedef int (*pair_pred)(const void *ctx, u32 i, u32 j);

static int emit_lists(u32 ntip, pair_pred pred, const void *ctx, u32 *counts, u32 *idx,
                      u64 cap, u64 *total, int nthreads) {
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 16)
    for (long i = 0; i < (long)ntip; i++) {
        u32 n = 0;
        for (u32 j = 0; j < ntip; j++) n += pred(ctx, (u32)i, j) ? 1u : 0u;
        counts[i] = n;
    }
    u64 tot = 0;
    for (u32 i = 0; i < ntip; i++) tot += counts[i];
    if (total) *total = tot;
    if (!idx) return ORACLE_OK;
    if (tot > cap) return ORACLE_ERANGE;
    u64 *off = (u64 *)malloc(sizeof(u64) * (ntip ? ntip : 1));
    if (!off) return ORACLE_ENOMEM;
    u64 acc = 0;
    for (u32 i = 0; i < ntip; i++) { off[i] = acc; acc += counts[i]; }
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 16)
    for (long i = 0; i < (long)ntip; i++) {
        u64 o = off[i];
        for (u32 j = 0; j < ntip; j++)
            if (pred(ctx, (u32)i, j)) idx[o++] = j;
    }
    free(off);
    return ORACLE_OK;
}

typedef struct { const u32 *bmat; u32 nrow, ntip; const float *wf; float radius; } RbCtx;
static int rb_pred(const void *p, u32 i, u32 j) {
    const RbCtx *c = (const RbCtx *)p;
    return radius_bit_score(c->bmat, c->nrow, c->ntip, c->wf, i, j) >= c->radius;
}

int oracle_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t *bmat,
                      const double *w, int32_t radius, uint32_t *counts,
                      uint32_t *idx, uint64_t idx_cap, uint64_t *total, int nthreads) {
    if (ntip == 0 || nrow == 0) return ORACLE_EINVAL;
    nthreads = nthreads_or_default(nthreads);
    float *wf = (float *)malloc(sizeof(float) * nrow * 32);
    if (!wf) return ORACLE_ENOMEM;
    for (u32 i = 0; i < nrow * 32; i++) wf[i] = (float)w[i];
    RbCtx c = {bmat, nrow, ntip, wf, (float)radius};
    int st = emit_lists(ntip, rb_pred, &c, counts, idx, idx_cap, total, nthreads);
    free(wf);
    return st;
}

/* radiusNeighborDNA (cu/radiusNeighborDNA.cu:27-87): low nibble of each
 * fasta2bin byte, count of positions whose nibbles intersect. */
static u32 dna_count(const u32 *raw, u32 nbinRaw, u32 q, u32 c) {
    const u32 *a = raw + (size_t)q * nbinRaw, *b = raw + (size_t)c * nbinRaw;
    u32 n = 0;
    for (u32 t = 0; t < nbinRaw; t++) {
        u32 v = a[t] & b[t] & 0x0F0F0F0Fu;
        n += ((v & 0xFFu) != 0) + ((v & 0xFF00u) != 0) + ((v & 0xFF0000u) != 0) + ((v & 0xFF000000u) != 0);
    }
    return n;
}

typedef struct { const u32 *raw; u32 nbinRaw; u32 radius; } RdCtx;
static int rd_pred(const void *p, u32 i, u32 j) {
    const RdCtx *c = (const RdCtx *)p;
    return dna_count(c->raw, c->nbinRaw, i, j) >= c->radius;
}

int oracle_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw,
                      uint32_t radius, uint32_t *counts, uint32_t *idx,
                      uint64_t idx_cap, uint64_t *total, int nthreads) {
    if (ntip == 0 || nbinRaw == 0) return ORACLE_EINVAL;
    RdCtx c = {raw, nbinRaw, radius};
    return emit_lists(ntip, rd_pred, &c, counts, idx, idx_cap, total, nthreads_or_default(nthreads));
}

/* tryRadius (cu/tryRadius.cu:26-50,122-158).  Threads past ntip in the last
 * 128-thread block score 0 and join the ballot, so a radius <= 0 adds
 * ceil(ntip/128)*128 - ntip to every count. */
int oracle_try_radius_bit(uint32_t nrow, uint32_t ntip, const uint32_t *bmat,
                          const double *w, int32_t radius, uint32_t nrep,
                          const uint32_t *qidx, uint32_t *counts, int nthreads) {
    if (ntip == 0 || nrow == 0) return ORACLE_EINVAL;
    nthreads = nthreads_or_default(nthreads);
    float *wf = (float *)malloc(sizeof(float) * nrow * 32);
    if (!wf) return ORACLE_ENOMEM;
    for (u32 i = 0; i < nrow * 32; i++) wf[i] = (float)w[i];
    const float r = (float)radius;
    const u32 pad = ((ntip + 127u) / 128u) * 128u - ntip;
    int bad = 0;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (long t = 0; t < (long)nrep; t++) {
        u32 q = qidx[t];
        if (q >= ntip) { bad = 1; continue; }
        u32 n = 0;
        for (u32 j = 0; j < ntip; j++) n += radius_bit_score(bmat, nrow, ntip, wf, q, j) >= r;
        if (0.0f >= r) n += pad;
        counts[t] = n;
    }
    free(wf);
    return bad ? ORACLE_ERANGE : ORACLE_OK;
}

/* tryRadiusDNA (cu/tryRadiusDNA.cu:45-74,139-148). */
int oracle_try_radius_dna(uint32_t ntip, uint32_t nbinRaw, const uint32_t *raw,
                          uint32_t radius, uint32_t nrep, const uint32_t *qidx,
                          uint32_t *counts, int nthreads) {
    if (ntip == 0 || nbinRaw == 0) return ORACLE_EINVAL;
    int bad = 0;
#pragma omp parallel for num_threads(nthreads_or_default(nthreads)) schedule(dynamic, 1)
    for (long t = 0; t < (long)nrep; t++) {
        u32 q = qidx[t];
        if (q >= ntip) { bad = 1; continue; }
        u32 n = 0;
        for (u32 j = 0; j < ntip; j++) n += dna_count(raw, nbinRaw, q, j) >= radius;
        counts[t] = n;
    }
    return bad ? ORACLE_ERANGE : ORACLE_OK;
}

/* ------------------------------------------------------------------ */
/* TransferDisStream (cu/TransferDisStream.cu:22-128,193-339).           */
/* The kernel reduces 8x8 tiles: for each x and each aligned group of 8  */
/* y rows it keeps A = min popc(x^y) and B = min popc(x^~y) separately    */
/* (absent rows contribute 32*ncol to both), then atomicMin(min(A,       */
/* B - (32*ncol - ntip))) with u32 wrap-around; symmetric for ymin over  */
/* groups of 8 x rows.  xmin/ymin start at 32*ncol.                      */
/* ------------------------------------------------------------------ */

static inline u32 xor_pop(const u32 *a, const u32 *b, u32 ncol) {
    u32 d = 0;
    for (u32 t = 0; t < ncol; t++) d += (u32)__builtin_popcount(a[t] ^ b[t]);
    return d;
}

static void tdis_side(u32 nA, u32 nB, u32 ncol, u32 ntip, const u32 *A, const u32 *B,
                      u32 *outmin, int nthreads) {
    const u32 full = 32u * ncol, pad = 32u * ncol - ntip;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 8)
    for (long a = 0; a < (long)nA; a++) {
        u32 best = full;
        for (u32 g = 0; g < nB; g += 8) {
            u32 mA = full, mB = full;
            for (u32 k = g; k < g + 8 && k < nB; k++) {
                u32 d = xor_pop(A + (size_t)a * ncol, B + (size_t)k * ncol, ncol);
                u32 comp = full - d;
                if (d < mA) mA = d;
                if (comp < mB) mB = comp;
            }
            u32 t2 = mB - pad;
            u32 v = mA > t2 ? t2 : mA;
            if (v < best) best = v;
        }
        outmin[a] = best;
    }
}

static void row_size(u32 n, u32 ncol, u32 ntip, const u32 *m, u32 *size) {
    for (u32 i = 0; i < n; i++) {
        u32 c = 0;
        for (u32 t = 0; t < ncol; t++) c += (u32)__builtin_popcount(m[(size_t)i * ncol + t]);
        if (c > ntip - c) c = ntip - c;
        size[i] = c;
    }
}

int oracle_transfer_dis(uint32_t nrow_y, uint32_t nrow_x, uint32_t ncol, uint32_t ntip,
                        const uint32_t *y, const uint32_t *x, uint32_t *ymin,
                        uint32_t *ysize, uint32_t *xmin, uint32_t *xsize, int nthreads) {
    if (ncol == 0) return ORACLE_EINVAL;
    nthreads = nthreads_or_default(nthreads);
    tdis_side(nrow_x, nrow_y, ncol, ntip, x, y, xmin, nthreads);
    tdis_side(nrow_y, nrow_x, ncol, ntip, y, x, ymin, nthreads);
    row_size(nrow_y, ncol, ntip, y, ysize);
    row_size(nrow_x, ncol, ntip, x, xsize);
    return ORACLE_OK;
}

/* ------------------------------------------------------------------------
 * Parsimony change counts (the reference's branch-length surrogate).
 * ancestralBitReverse, src/functions.cpp:3478-3542: a bottom-up pass over the
 * edges in reverse order keeps per internal node a state (AND of the
 * children), a bistate (AND of the children's bistates; tips 0) and a
 * conflict mask (bits where a child differs from the AND so far and neither
 * side is bistate); a child's conflict bits are folded into its state and
 * bistate when its parent edge is reached.  The root then drops its
 * conflict and bistate bits.  A pre-order pass resolves every internal
 * child's bistate bits from its parent ((s & ~bs) | (parent & bs),
 * calcDesStateBitReverse :3464-3476) and counts the differing bits per edge
 * (countBitEvo :3005-3015).
 */
int oracle_ancestral_bit(uint32_t ntip, uint32_t nnode, uint32_t nbin, const uint32_t *mat,
                         uint32_t nedge, const uint32_t *edge, uint32_t *state, uint32_t *bis,
                         uint32_t *len) {
    if (!mat || !edge || !state || !bis || !len || nnode == 0) return ORACLE_EINVAL;
    u32 *conf = (u32 *)calloc((size_t)nnode * nbin, sizeof(u32));
    if (!conf) return ORACLE_ENOMEM;
    for (size_t i = 0; i < (size_t)nnode * nbin; i++) { state[i] = 0xFFFFFFFFu; bis[i] = 0xFFFFFFFFu; }
    for (long i = (long)nedge - 1; i >= 0; i--) {
        const u32 a = edge[2 * i], d = edge[2 * i + 1];
        if (a < ntip || a >= ntip + nnode || d >= ntip + nnode) { free(conf); return ORACLE_EINVAL; }
        u32 *sa = state + (size_t)(a - ntip) * nbin, *ba = bis + (size_t)(a - ntip) * nbin;
        u32 *ca = conf + (size_t)(a - ntip) * nbin;
        for (u32 j = 0; j < nbin; j++) {
            u32 s2, bs2;
            if (d < ntip) {
                s2 = mat[(size_t)d * nbin + j];
                bs2 = 0;
            } else {
                u32 *sd = state + (size_t)(d - ntip) * nbin, *bd = bis + (size_t)(d - ntip) * nbin;
                const u32 cd = conf[(size_t)(d - ntip) * nbin + j];
                sd[j] |= cd;
                bd[j] |= cd;
                s2 = sd[j];
                bs2 = bd[j];
            }
            const u32 s1 = sa[j], bs1 = ba[j];
            sa[j] = s1 & s2;
            ba[j] &= bs2;
            ca[j] |= (s1 ^ s2) & ~(bs1 | bs2);
        }
    }
    for (u32 j = 0; j < nbin; j++) state[j] &= ~(conf[j] | bis[j]);
    for (u32 i = 0; i < nedge; i++) {
        const u32 a = edge[2 * i], d = edge[2 * i + 1];
        const u32 *sa = state + (size_t)(a - ntip) * nbin;
        u32 cnt = 0;
        if (d < ntip) {
            for (u32 j = 0; j < nbin; j++) cnt += (u32)__builtin_popcount(sa[j] ^ mat[(size_t)d * nbin + j]);
        } else {
            u32 *sd = state + (size_t)(d - ntip) * nbin;
            const u32 *bd = bis + (size_t)(d - ntip) * nbin;
            for (u32 j = 0; j < nbin; j++) {
                sd[j] = (sd[j] & ~bd[j]) | (sa[j] & bd[j]);
                cnt += (u32)__builtin_popcount(sa[j] ^ sd[j]);
            }
        }
        len[i] = cnt;
    }
    free(conf);
    return ORACLE_OK;
}

/* charAncestralEC, src/functions.cpp:3085-3150: node sizes and the largest
 * child size bottom-up; then, over the edges in reverse order, a child that
 * passes the size rule (minRatio * size >= largest sibling size, or size >=
 * minSize) sets each unknown (-1) site of its parent to its own value, and a
 * known site that disagrees with a known child value becomes 0.  Edge
 * lengths count the sites where both ends are known and differ
 * (countCharEvo :3074-3082). */
int oracle_ancestral_char(uint32_t ntip, uint32_t nnode, uint32_t nsite, const int32_t *mat,
                          uint32_t nedge, const uint32_t *edge, const uint32_t *tipSize,
                          float minSize, float minRatio, int32_t *state, uint32_t *len) {
    if (!mat || !edge || !state || !len || !tipSize || nnode == 0) return ORACLE_EINVAL;
    int32_t *nsz = (int32_t *)calloc(nnode, sizeof(int32_t)), *mx = (int32_t *)calloc(nnode, sizeof(int32_t));
    if (!nsz || !mx) { free(nsz); free(mx); return ORACLE_ENOMEM; }
    for (long i = (long)nedge - 1; i >= 0; i--) {
        const u32 a = edge[2 * i], d = edge[2 * i + 1];
        if (a < ntip || a >= ntip + nnode || d >= ntip + nnode) { free(nsz); free(mx); return ORACLE_EINVAL; }
        const int32_t sd = d < ntip ? (int32_t)tipSize[d] : nsz[d - ntip];
        nsz[a - ntip] += sd;
        if (mx[a - ntip] < sd) mx[a - ntip] = sd;
    }
    for (size_t i = 0; i < (size_t)nnode * nsite; i++) state[i] = -1;
    for (long i = (long)nedge - 1; i >= 0; i--) {
        const u32 a = edge[2 * i], d = edge[2 * i + 1];
        const int32_t sd = d < ntip ? (int32_t)tipSize[d] : nsz[d - ntip];
        if (!(minRatio * (float)sd >= (float)mx[a - ntip] || (float)sd >= minSize)) continue;
        int32_t *pa = state + (size_t)(a - ntip) * nsite;
        const int32_t *pd = d < ntip ? mat + (size_t)d * nsite : state + (size_t)(d - ntip) * nsite;
        for (u32 j = 0; j < nsite; j++) {
            if (pa[j] == -1) pa[j] = pd[j];
            else if (pa[j] != pd[j] && pd[j] != -1) pa[j] = 0;
        }
    }
    for (u32 i = 0; i < nedge; i++) {
        const u32 a = edge[2 * i], d = edge[2 * i + 1];
        const int32_t *pa = state + (size_t)(a - ntip) * nsite;
        const int32_t *pd = d < ntip ? mat + (size_t)d * nsite : state + (size_t)(d - ntip) * nsite;
        u32 cnt = 0;
        for (u32 j = 0; j < nsite; j++) cnt += pa[j] >= 0 && pd[j] >= 0 && pa[j] != pd[j];
        len[i] = cnt;
    }
    free(nsz);
    free(mx);
    return ORACLE_OK;
}

/* ------------------------------------------------------------------------
 * tipMerge (cu/tipMerge.cu:130-461).  Rows are visited in chunks of 131072
 * candidate columns (CACHEMAX): for chunk [c0, c1) every row j < c1, in
 * increasing order, takes the neighbours k of its list with max(c0, j+1) <=
 * k < c1, keeps those that pass the reference's filter (:366-370: the root
 * of j's category against transitionRoot(transition, k), k used as a
 * category index), counts |N(j) n N(k)| for each (sharedIdxKernel :26-128,
 * an intersection of the two ascending lists) and then, in list order,
 * merges categories when the count exceeds pShared times either list's
 * length (:403-425).  Untouched rows get new categories in row order
 * (:446-456). */
static int tm_root(const int *transition, int idx) {
    if (idx == -1) return -1;
    int r = idx;
    while (transition[r] != r && transition[r] != -1) r = transition[r];
    return r;
}

static u32 tm_shared(const u32 *a, u32 na, const u32 *b, u32 nb) {
    u32 i = 0, j = 0, n = 0;
    while (i < na && j < nb) {
        if (a[i] < b[j]) i++;
        else if (a[i] > b[j]) j++;
        else { n++; i++; j++; }
    }
    return n;
}

int oracle_tip_merge(uint32_t ntip, const uint32_t *counts, const uint32_t *idx, double pShared,
                     int32_t *member) {
    if (!counts || !member || ntip == 0) return ORACLE_EINVAL;
    const u32 kCache = 1024u * 128u, kMaxNeighbor = 1024u * 1024u;
    u64 *off = (u64 *)malloc(sizeof(u64) * (ntip + 1));
    u32 *so = (u32 *)malloc(sizeof(u32) * ntip);
    int *tr = (int *)malloc(sizeof(int) * ntip);
    u32 *run = (u32 *)malloc(sizeof(u32) * (ntip ? ntip : 1));
    u32 *sh = (u32 *)malloc(sizeof(u32) * (ntip ? ntip : 1));
    if (!off || !so || !tr || !run || !sh) { free(off); free(so); free(tr); free(run); free(sh); return ORACLE_ENOMEM; }
    off[0] = 0;
    int st = ORACLE_OK;
    for (u32 i = 0; i < ntip; i++) {
        if (counts[i] > kMaxNeighbor) { st = ORACLE_ERANGE; goto done; }
        off[i + 1] = off[i] + counts[i];
    }
    for (u32 i = 0; i < ntip; i++) {
        u32 j = 0;
        while (j < counts[i] && idx[off[i] + j] <= i) j++;
        so[i] = j;
        member[i] = -1;
        tr[i] = -1;
    }
    int ncat = 0;
    for (u32 c0 = 0; c0 < ntip; c0 += kCache) {
        const u32 c1 = c0 + kCache < ntip ? c0 + kCache : ntip;
        for (u32 j = 0; j < c1; j++) {
            int root1 = member[j];
            if (root1 != -1) root1 = tm_root(tr, root1);
            u32 nrun = 0;
            const u32 *lj = idx + off[j];
            for (u32 k = so[j]; k < counts[j]; k++) {
                const u32 t = lj[k];
                if (t >= c1) { so[j] = k; break; }
                if (t >= c0 && (root1 == -1 || root1 != tm_root(tr, (int)t))) run[nrun++] = t;
            }
            if (!nrun) continue;
            for (u32 k = 0; k < nrun; k++) sh[k] = tm_shared(lj, counts[j], idx + off[run[k]], counts[run[k]]);
            for (u32 k = 0; k < nrun; k++) {
                const u32 t = run[k];
                if ((double)sh[k] > counts[j] * pShared || (double)sh[k] > counts[t] * pShared) {
                    const int root2 = tm_root(tr, member[t]);
                    if (root1 == -1) {
                        if (root2 == -1) {
                            root1 = ncat;
                            tr[ncat] = ncat;
                            member[j] = ncat;
                            member[t] = ncat;
                            ncat++;
                        } else {
                            root1 = root2;
                            member[j] = root2;
                        }
                    } else {
                        if (root2 == -1) {
                            member[t] = root1;
                        } else {
                            tr[root1] = root2;
                            member[j] = root2;
                            root1 = root2;
                        }
                    }
                }
            }
        }
    }
    for (u32 i = 0; i < ntip; i++) member[i] = member[i] == -1 ? ncat++ : tm_root(tr, member[i]);
done:
    free(off); free(so); free(tr); free(run); free(sh);
    return st;
}

/* ------------------------------------------------------------------------
 * nodeDesBig (src/functions.cpp:1277-1366): over the edges in reverse order,
 * a tip child sets its bit in the parent's row and adds 1 to its size; an
 * internal child adds its size and ORs its row into the parent's, and its
 * own row is written out then.  The reference keeps the open rows in 8192
 * cache slots and stops with "Run out of cache!" when more are open.  The
 * returned sizes are those of internal nodes 1..nnode-1, last node first. */
int oracle_node_des(uint32_t ntip, uint32_t nnode, uint32_t nedge, const uint32_t *edge,
                    uint32_t *rows_out, int32_t *sizes_out) {
    if (!edge || !rows_out || !sizes_out || nnode == 0 || ntip == 0) return ORACLE_EINVAL;
    const u32 nbin = ((ntip - 1) >> 5) + 1, kCache = 8192;
    u32 *bits = (u32 *)calloc((size_t)nnode * nbin, sizeof(u32));
    int32_t *size = (int32_t *)calloc(nnode, sizeof(int32_t));
    char *open = (char *)calloc(nnode, 1);
    if (!bits || !size || !open) { free(bits); free(size); free(open); return ORACLE_ENOMEM; }
    int st = ORACLE_OK;
    u32 nUse = 0, r = 0;
    for (long i = (long)nedge - 1; i >= 0; i--) {
        const u32 a = edge[2 * i], d = edge[2 * i + 1];
        if (a < ntip || a >= ntip + nnode || d >= ntip + nnode) { st = ORACLE_EINVAL; break; }
        const u32 ai = a - ntip;
        if (!open[ai]) {
            if (nUse == kCache) { st = ORACLE_ERANGE; break; }
            open[ai] = 1;
            nUse++;
        }
        if (d < ntip) {
            size[ai]++;
            bits[(size_t)ai * nbin + (d >> 5)] |= 1u << (d & 31);
        } else {
            const u32 di = d - ntip;
            size[ai] += size[di];
            for (u32 x = 0; x < nbin; x++) bits[(size_t)ai * nbin + x] |= bits[(size_t)di * nbin + x];
            memcpy(rows_out + (size_t)r * nbin, bits + (size_t)di * nbin, sizeof(u32) * nbin);
            r++;
            open[di] = 0;
            nUse--;
        }
    }
    if (st == ORACLE_OK)
        for (u32 i = 1; i < nnode; i++) sizes_out[nnode - 1 - i] = size[i];
    free(bits); free(size); free(open);
    return st;
}

/* ------------------------------------------------------------------------
 * approximateCompare2_AVX2 (src/functions.cpp:5450-5600).  The query tree's
 * edges are visited in reverse order.  A tip child sets its bit in the
 * parent's open row and its stop node becomes its parent in the reference
 * tree.  An internal child d ORs its row into the parent's, then from the
 * stop node of each of its children (in edge order) walks up the reference
 * tree while the node is not the root and the previous comparison left at
 * most size(d) * threshold tips outside d (binary32 product): at each node it
 * takes the XOR distance to d and the count of the node's tips missing
 * from d, lowers the node's best distance (ties go to the later d) and d's
 * best distance (ties go to the later node, which also becomes d's stop
 * node).  d's stop node starts as its first child's.  The reference keeps
 * the open rows in cacheSize slots and stops when more are needed. */
int oracle_approx_compare(uint32_t ntip, uint32_t nnode1, uint32_t nbin, const uint32_t *clade, uint32_t nedge1,
                          const uint32_t *edge1, uint32_t nedge2, const uint32_t *edge2, uint32_t nnode2,
                          uint32_t cacheSize, float threshold, int32_t *ref2qry, int32_t *qry2ref) {
    if (!clade || !edge1 || !edge2 || !ref2qry || !qry2ref || ntip == 0 || nnode1 == 0 || nnode2 == 0 ||
        nbin != ((ntip - 1) >> 5) + 1)
        return ORACLE_EINVAL;
    const u32 n1 = ntip + nnode1, n2 = ntip + nnode2;
    int32_t *par1 = (int32_t *)malloc(sizeof(int32_t) * n1);
    u32 *stop = (u32 *)malloc(sizeof(u32) * n2);
    int32_t *size2 = (int32_t *)calloc(n2, sizeof(int32_t));
    u32 *bits = (u32 *)calloc((size_t)nnode2 * nbin, sizeof(u32));
    char *open = (char *)calloc(nnode2, 1);
    u32 *kidOff = (u32 *)calloc(nnode2 + 1, sizeof(u32));
    u32 *kids = (u32 *)malloc(sizeof(u32) * (nedge2 ? nedge2 : 1));
    u32 *fill = (u32 *)calloc(nnode2, sizeof(u32));
    int32_t *d1 = (int32_t *)malloc(sizeof(int32_t) * nnode1), *m1 = (int32_t *)calloc(nnode1, sizeof(int32_t));
    int32_t *d2 = (int32_t *)malloc(sizeof(int32_t) * nnode2), *m2 = (int32_t *)calloc(nnode2, sizeof(int32_t));
    int st = ORACLE_OK;
    if (!par1 || !stop || !size2 || !bits || !open || !kidOff || !kids || !fill || !d1 || !m1 || !d2 || !m2) {
        st = ORACLE_ENOMEM;
        goto done;
    }
    for (u32 v = 0; v < n1; v++) par1[v] = -1;
    for (u32 i = 0; i < nedge1; i++) {
        if (edge1[2 * i] >= n1 || edge1[2 * i + 1] >= n1) { st = ORACLE_EINVAL; goto done; }
        par1[edge1[2 * i + 1]] = (int32_t)edge1[2 * i];
    }
    for (u32 i = 0; i < nedge2; i++) {
        const u32 a = edge2[2 * i], d = edge2[2 * i + 1];
        if (a < ntip || a >= n2 || d >= n2) { st = ORACLE_EINVAL; goto done; }
        kidOff[a - ntip + 1]++;
    }
    for (u32 i = 0; i < nnode2; i++) kidOff[i + 1] += kidOff[i];
    for (u32 i = 0; i < nedge2; i++) {
        const u32 ai = edge2[2 * i] - ntip;
        kids[kidOff[ai] + fill[ai]++] = edge2[2 * i + 1];
    }
    for (u32 v = 0; v < n2; v++) stop[v] = ntip;
    for (u32 i = 0; i < nnode1; i++) d1[i] = (int32_t)(2 * ntip);
    for (u32 i = 0; i < nnode2; i++) d2[i] = (int32_t)(2 * ntip);
    u32 nUse = 0;
    for (long i = (long)nedge2 - 1; i >= 0; i--) {
        const u32 a = edge2[2 * i], d = edge2[2 * i + 1], ai = a - ntip;
        if (!open[ai]) {
            if (nUse == cacheSize) { st = ORACLE_ERANGE; goto done; }
            open[ai] = 1;
            nUse++;
        }
        u32 *ra = bits + (size_t)ai * nbin;
        if (d < ntip) {
            size2[d] = 1;
            size2[a]++;
            ra[d >> 5] |= 1u << (d & 31);
            stop[d] = (u32)par1[d];
            continue;
        }
        const u32 di = d - ntip;
        const u32 *rd = bits + (size_t)di * nbin;
        size2[a] += size2[d];
        for (u32 x = 0; x < nbin; x++) ra[x] |= rd[x];
        const u32 k0 = kidOff[di], k1 = kidOff[di + 1];
        stop[d] = stop[kids[k0]];
        int32_t best = (int32_t)(2 * ntip);
        const float lim = (float)size2[d] * threshold;
        for (u32 k = k0; k < k1; k++) {
            u32 cur = stop[kids[k]];
            int32_t nLarger = 0;
            while (cur > ntip && (float)nLarger <= lim) {
                const u32 t = nnode1 - 1 - (cur - ntip);
                const u32 *rc = clade + (size_t)t * nbin;
                int32_t xr = 0;
                nLarger = 0;
                for (u32 x = 0; x < nbin; x++) {
                    xr += __builtin_popcount(rc[x] ^ rd[x]);
                    nLarger += __builtin_popcount(rc[x] & ~rd[x]);
                }
                if (d1[t] >= xr) { d1[t] = xr; m1[t] = (int32_t)d + 1; }
                if (best >= xr) {
                    best = xr;
                    stop[d] = cur;
                    d2[di] = xr;
                    m2[di] = (int32_t)cur + 1;
                }
                cur = (u32)par1[cur];
            }
        }
        memset(bits + (size_t)di * nbin, 0, sizeof(u32) * nbin);
        open[di] = 0;
        nUse--;
    }
    ref2qry[0] = (int32_t)ntip + 1;
    ref2qry[1] = 0;
    for (u32 i = 1; i < nnode1; i++) {
        ref2qry[2 * i] = m1[nnode1 - 1 - i];
        ref2qry[2 * i + 1] = d1[nnode1 - 1 - i];
    }
    for (u32 i = 0; i < nnode2; i++) {
        qry2ref[3 * i] = m2[i];
        qry2ref[3 * i + 1] = d2[i];
        qry2ref[3 * i + 2] = size2[ntip + i];
    }
    qry2ref[0] = (int32_t)ntip + 1;
    qry2ref[1] = 0;
done:
    free(par1); free(stop); free(size2); free(bits); free(open); free(kidOff); free(kids); free(fill);
    free(d1); free(m1); free(d2); free(m2);
    return st;
}

/* ------------------------------------------------------------------ */
/* FP64 log-likelihoods for branch-length checks at full size.          */
/* CasPhy has no likelihood code; these restate Felsenstein (1981)      */
/* pruning in double precision, like oracle/felsenstein.py (which the   */
/* CPU tests compare them with), but site-blocked in C so that trees    */
/* of 10^5 tips take seconds.  Tree: edge nedge x 2 (parent, child),    */
/* tips 0..ntip-1, every internal node with two children, the root the  */
/* node that is no child.                                               */
/* ------------------------------------------------------------------ */

typedef struct {
    u32 nn, root;
    u32 *kid;   /* nn x 2 */
    u32 *eoc;   /* edge of child, per node */
    u32 *post;  /* internal nodes, children before parents */
    u32 npost;
} FelTree;

static int fel_tree(u32 ntip, u32 nedge, const u32 *edge, FelTree *T) {
    const u32 nn = nedge + 1;
    T->nn = nn;
    T->kid = (u32 *)malloc(sizeof(u32) * 2 * nn);
    T->eoc = (u32 *)malloc(sizeof(u32) * nn);
    T->post = (u32 *)malloc(sizeof(u32) * nn);
    u32 *nk = (u32 *)calloc(nn, sizeof(u32));
    u32 *stack = (u32 *)malloc(sizeof(u32) * nn);
    unsigned char *isChild = (unsigned char *)calloc(nn, 1);
    if (!T->kid || !T->eoc || !T->post || !nk || !stack || !isChild) { free(nk); free(stack); free(isChild); return ORACLE_ENOMEM; }
    int st = ORACLE_OK;
    for (u32 e = 0; e < nedge; e++) {
        const u32 p = edge[2 * e], c = edge[2 * e + 1];
        if (p >= nn || c >= nn || p < ntip || nk[p] >= 2 || isChild[c]) { st = ORACLE_EINVAL; goto out; }
        T->kid[2 * p + nk[p]++] = c;
        T->eoc[c] = e;
        isChild[c] = 1;
    }
    T->root = nn;
    for (u32 v = 0; v < nn; v++)
        if (!isChild[v]) { if (T->root != nn) { st = ORACLE_EINVAL; goto out; } T->root = v; }
    for (u32 v = ntip; v < nn; v++) if (nk[v] != 2) { st = ORACLE_EINVAL; goto out; }
    /* reverse of a pre-order walk: children before parents */
    u32 sp = 0, n = 0;
    stack[sp++] = T->root;
    while (sp) {
        const u32 v = stack[--sp];
        if (v < ntip) continue;
        T->post[n++] = v;
        stack[sp++] = T->kid[2 * v];
        stack[sp++] = T->kid[2 * v + 1];
    }
    for (u32 i = 0; i < n / 2; i++) { const u32 x = T->post[i]; T->post[i] = T->post[n - 1 - i]; T->post[n - 1 - i] = x; }
    T->npost = n;
out:
    free(nk); free(stack); free(isChild);
    return st;
}

static void fel_tree_free(FelTree *T) { free(T->kid); free(T->eoc); free(T->post); }

#define FEL_SB 16u /* sites per block */

/* HKY85 (Hasegawa, Kishino & Yano 1985) on fasta2bin nibbles (bit 0 A,
 * 1 T, 2 C, 3 G; several bits ambiguous, none missing).  P(t) = expm(Q t)
 * with Q normalised to one substitution per unit time, from the eigen
 * decomposition of the symmetrised Q (Q is reversible). */
static void hky_Q(double kappa, const double *pi, double Q[4][4]) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) Q[i][j] = i == j ? 0.0 : pi[j];
    Q[0][3] *= kappa; Q[3][0] *= kappa; Q[1][2] *= kappa; Q[2][1] *= kappa;
    double mu = 0;
    for (int i = 0; i < 4; i++) {
        double s = 0;
        for (int j = 0; j < 4; j++) s += Q[i][j];
        Q[i][i] = -s;
        mu += pi[i] * s;
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) Q[i][j] /= mu;
}

/* Jacobi eigen decomposition of a symmetric 4x4 matrix: A = V diag(w) V^T. */
static void jacobi4(double A[4][4], double w[4], double V[4][4]) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) V[i][j] = i == j;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0;
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++) off += A[i][j] * A[i][j];
        if (off < 1e-300) break;
        for (int p = 0; p < 4; p++)
            for (int q = p + 1; q < 4; q++) {
                if (fabs(A[p][q]) < 1e-300) continue;
                const double th = (A[q][q] - A[p][p]) / (2 * A[p][q]);
                const double tt = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1));
                const double c = 1 / sqrt(tt * tt + 1), s = tt * c;
                for (int k = 0; k < 4; k++) {
                    const double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 4; k++) {
                    const double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 4; k++) {
                    const double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 4; i++) w[i] = A[i][i];
}

int oracle_loglik_hky85(uint32_t ntip, uint32_t nedge, const uint32_t *edge, const double *t, uint32_t nsite,
                        const uint32_t *codes, const double *weights, double kappa, const double *pi, double *ll,
                        int nthreads) {
    FelTree T;
    memset(&T, 0, sizeof(T));
    int st = fel_tree(ntip, nedge, edge, &T);
    if (st) { fel_tree_free(&T); return st; }
    double Q[4][4], S[4][4], w[4], V[4][4], sq[4];
    hky_Q(kappa, pi, Q);
    for (int i = 0; i < 4; i++) sq[i] = sqrt(pi[i]);
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) S[i][j] = sq[i] * Q[i][j] / sq[j];
    jacobi4(S, w, V);
    /* P(t) for every edge: P = D^-1/2 V exp(w t) V^T D^1/2 */
    double *P = (double *)malloc(sizeof(double) * 16 * (nedge ? nedge : 1));
    if (!P) { fel_tree_free(&T); return ORACLE_ENOMEM; }
    for (u32 e = 0; e < nedge; e++)
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++) {
                double s = 0;
                for (int k = 0; k < 4; k++) s += V[i][k] * exp(w[k] * t[e]) * V[j][k];
                P[16 * e + 4 * i + j] = s * sq[j] / sq[i];
            }
    const u32 nn = T.nn, nblk = (nsite + FEL_SB - 1) / FEL_SB;
    double total = 0;
    nthreads = nthreads_or_default(nthreads);
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
    {
        double *L = (double *)malloc(sizeof(double) * (size_t)nn * FEL_SB * 4);
        double *lsc = (double *)malloc(sizeof(double) * (size_t)nn * FEL_SB);
#pragma omp for schedule(dynamic, 1)
        for (long blk = 0; blk < (long)nblk; blk++) {
            const u32 s0 = (u32)blk * FEL_SB, ns = nsite - s0 < FEL_SB ? nsite - s0 : FEL_SB;
            for (u32 v = 0; v < ntip; v++)
                for (u32 k = 0; k < ns; k++) {
                    const u32 nib = codes[(size_t)v * nsite + s0 + k] & 0xFu;
                    for (int i = 0; i < 4; i++) L[((size_t)v * FEL_SB + k) * 4 + i] = nib ? (double)((nib >> i) & 1u) : 1.0;
                    lsc[(size_t)v * FEL_SB + k] = 0;
                }
            for (u32 x = 0; x < T.npost; x++) {
                const u32 v = T.post[x];
                for (u32 k = 0; k < ns; k++) {
                    double acc[4] = {1, 1, 1, 1}, sc = 0;
                    for (int h = 0; h < 2; h++) {
                        const u32 c = T.kid[2 * v + h];
                        const double *Pc = P + 16 * T.eoc[c], *Lc = L + ((size_t)c * FEL_SB + k) * 4;
                        for (int i = 0; i < 4; i++)
                            acc[i] *= Pc[4 * i] * Lc[0] + Pc[4 * i + 1] * Lc[1] + Pc[4 * i + 2] * Lc[2] + Pc[4 * i + 3] * Lc[3];
                        sc += lsc[(size_t)c * FEL_SB + k];
                    }
                    double m = acc[0];
                    for (int i = 1; i < 4; i++) m = acc[i] > m ? acc[i] : m;
                    if (m <= 0) m = 1;
                    for (int i = 0; i < 4; i++) L[((size_t)v * FEL_SB + k) * 4 + i] = acc[i] / m;
                    lsc[(size_t)v * FEL_SB + k] = sc + log(m);
                }
            }
            for (u32 k = 0; k < ns; k++) {
                const double *Lr = L + ((size_t)T.root * FEL_SB + k) * 4;
                const double site = log(pi[0] * Lr[0] + pi[1] * Lr[1] + pi[2] * Lr[2] + pi[3] * Lr[3]) +
                                    lsc[(size_t)T.root * FEL_SB + k];
                total += (weights ? weights[s0 + k] : 1.0) * site;
            }
        }
        free(L); free(lsc);
    }
    *ll = total;
    free(P);
    fel_tree_free(&T);
    return ORACLE_OK;
}

/* Irreversible edit model: per site state 0 = unedited, 1..K alleles;
 * P(0->0) = exp(-r t), P(0->a) = q_a (1 - exp(-r t)), P(a->b) = [a == b];
 * the root is unedited.  Tip codes (.tbmat): 0 missing, 1 unedited, c >= 2
 * allele c-1.  Because alleles never change, a node's partial is non-zero
 * on state 0 and on at most one allele: the one its subtree's non-missing
 * tips share (none when they disagree or one is unedited; every allele,
 * with one common value, when all its tips are missing).  The partial is
 * kept as (L0, La, allele) with allele -1 none, 0 every allele, a >= 1. */
int oracle_loglik_irreversible(uint32_t ntip, uint32_t nedge, const uint32_t *edge, const double *t, uint32_t nsite,
                               const uint32_t *codes, const double *weights, uint32_t K, const double *q,
                               double rate, double *ll, int nthreads) {
    FelTree T;
    memset(&T, 0, sizeof(T));
    int st = fel_tree(ntip, nedge, edge, &T);
    if (st) { fel_tree_free(&T); return st; }
    const u32 nn = T.nn, nblk = (nsite + FEL_SB - 1) / FEL_SB;
    double total = 0;
    nthreads = nthreads_or_default(nthreads);
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
    {
        double *L0 = (double *)malloc(sizeof(double) * (size_t)nn * FEL_SB);
        double *La = (double *)malloc(sizeof(double) * (size_t)nn * FEL_SB);
        double *lsc = (double *)malloc(sizeof(double) * (size_t)nn * FEL_SB);
        int *A = (int *)malloc(sizeof(int) * (size_t)nn * FEL_SB);
#pragma omp for schedule(dynamic, 1)
        for (long blk = 0; blk < (long)nblk; blk++) {
            const u32 s0 = (u32)blk * FEL_SB, ns = nsite - s0 < FEL_SB ? nsite - s0 : FEL_SB;
            for (u32 v = 0; v < ntip; v++)
                for (u32 k = 0; k < ns; k++) {
                    const u32 c = codes[(size_t)v * nsite + s0 + k];
                    const size_t i = (size_t)v * FEL_SB + k;
                    lsc[i] = 0;
                    if (c == 0) { L0[i] = 1; La[i] = 1; A[i] = 0; }
                    else if (c == 1) { L0[i] = 1; La[i] = 0; A[i] = -1; }
                    else { L0[i] = 0; La[i] = 1; A[i] = (int)c - 1; }
                }
            for (u32 x = 0; x < T.npost; x++) {
                const u32 v = T.post[x];
                for (u32 k = 0; k < ns; k++) {
                    const size_t iv = (size_t)v * FEL_SB + k;
                    double l0 = 1, la = 1, sc = 0;
                    int a = 0;
                    for (int h = 0; h < 2; h++) {
                        const u32 c = T.kid[2 * v + h];
                        const size_t ic = (size_t)c * FEL_SB + k;
                        const double p = exp(-rate * t[T.eoc[c]]);
                        /* sum over the child's alleles of P(0->b) L_c(b) */
                        double edited = 0;
                        if (A[ic] == 0) edited = (1 - p) * La[ic];
                        else if (A[ic] > 0) edited = (1 - p) * q[(size_t)(s0 + k) * (K + 1) + (u32)A[ic]] * La[ic];
                        l0 *= p * L0[ic] + edited;
                        /* alleles pass unchanged: the sets intersect */
                        if (A[ic] < 0 || a < 0) { a = -1; la = 0; }
                        else if (A[ic] == 0) la *= La[ic];
                        else if (a == 0 || a == A[ic]) { a = A[ic]; la *= La[ic]; }
                        else { a = -1; la = 0; }
                        sc += lsc[ic];
                    }
                    double m = l0 > la ? l0 : la;
                    if (m <= 0) m = 1;
                    L0[iv] = l0 / m;
                    La[iv] = la / m;
                    A[iv] = a;
                    lsc[iv] = sc + log(m);
                }
            }
            for (u32 k = 0; k < ns; k++) {
                const size_t ir = (size_t)T.root * FEL_SB + k;
                total += (weights ? weights[s0 + k] : 1.0) * (log(L0[ir]) + lsc[ir]);
            }
        }
        free(L0); free(La); free(lsc); free(A);
    }
    *ll = total;
    fel_tree_free(&T);
    return ORACLE_OK;
}
