/*
 * CPU restatement of EagleImp's data-parallel hot path -- TEST ORACLE.
 * See eimp_oracle.h for the contract.  Test infrastructure only: the product
 * never calls this code.  The phasing beam lives in eimp_oracle_beam.c.
 */
#include "eimp_oracle.h"

#include <stdlib.h>
#include <string.h>

size_t eo_W(size_t nbits) { return ((nbits + 511) / 512) * 8; }

static inline int popc64(uint64_t x) { return __builtin_popcountll(x); }
static inline int getbit(const uint64_t *v, size_t i) { return (int)((v[i >> 6] >> (i & 63)) & 1u); }
static inline void setbit(uint64_t *v, size_t i) { v[i >> 6] |= 1ull << (i & 63); }

/* ---------------------------------------------------------------- a1 + a2 */

typedef struct { uint64_t key; } eo_key;

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}
static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* Target.cpp:779-875: all haps when K >= Nrefhaps; otherwise the K smallest
 * pairs (nerr, index) -- std::sort of pairs orders ties by index -- then the
 * chosen indices ascending (Target.cpp:847). */
void eo_besthaps(const uint64_t *gtw, const uint64_t *hapmajor, size_t nhaps, size_t wM,
                 size_t K, int64_t *besthaps, uint32_t *nerr_out) {
    uint64_t *keys = (uint64_t *)malloc(nhaps * sizeof(uint64_t));
    for (size_t h = 0; h < nhaps; h++) {
        const uint64_t *row = hapmajor + h * wM;
        uint32_t nerr = 0;
        for (size_t w = 0; w < wM; w++)   /* Datatypes.cpp:111-114 */
            nerr += (uint32_t)popc64((gtw[2 * w] & row[w]) | (gtw[2 * w + 1] & ~row[w]));
        if (nerr_out) nerr_out[h] = nerr;
        keys[h] = ((uint64_t)nerr << 32) | (uint64_t)h;
    }
    if (K >= nhaps) {
        for (size_t k = 0; k < nhaps; k++) besthaps[k] = (int64_t)k;
    } else {
        qsort(keys, nhaps, sizeof(uint64_t), cmp_u64);
        for (size_t k = 0; k < K; k++) besthaps[k] = (int64_t)(keys[k] & 0xffffffffu);
        qsort(besthaps, K, sizeof(int64_t), cmp_i64);
    }
    free(keys);
}

/* ---------------------------------------------------------------- a3 */

void eo_monos(const uint64_t *hapmajor, size_t wM, size_t M, const int64_t *besthaps, size_t K,
              uint64_t *monos) {
    /* Target.cpp:878-897: every site < M starts as mono (bits >= M are 0,
     * Datatypes.h:344-356), then one XNOR-AND per consecutive best hap pair */
    for (size_t w = 0; w < wM; w++) {
        size_t lo = w * 64;
        monos[w] = lo + 64 <= M ? ~0ull : (lo >= M ? 0ull : ((1ull << (M - lo)) - 1));
    }
    for (size_t k = 1; k < K; k++) {
        const uint64_t *a = hapmajor + (size_t)besthaps[k - 1] * wM;
        const uint64_t *b = hapmajor + (size_t)besthaps[k] * wM;
        for (size_t w = 0; w < wM; w++) monos[w] &= ~(a[w] ^ b[w]);
    }
}

long eo_calllocs(const uint8_t *gt, const uint64_t *monos, const float *cm, size_t M,
                 float cMmaxsplit, int64_t *splits, int64_t *calls, size_t *ncalls, float *cmdiffs) {
    /* Target.cpp:900-950 */
    size_t S = 0, C = 0;
    float last = cm[0];
    size_t m;
    for (m = 0; m < M; m++)
        if (gt[m] == 1) break;               /* first het, mono or not (:907-912) */
    for (; m < M; m++) {
        if (!getbit(monos, m) && gt[m] != 3 && (gt[m] == 1 || cm[m] - last > cMmaxsplit)) {
            if (gt[m] == 1) calls[C++] = (int64_t)S;
            splits[S++] = (int64_t)m;
            last = cm[m];
        }
    }
    *ncalls = C;
    if (S == 0) return 0;
    if (C == 0) return 0;                    /* :927-932 */
    S = (size_t)calls[C - 1] + 1;            /* :936-937 */
    cmdiffs[0] = cm[splits[0]] - cm[0];
    for (size_t i = 1; i < S; i++) cmdiffs[i] = cm[splits[i]] - cm[splits[i - 1]];
    cmdiffs[S] = cm[M - 1] - cm[splits[S - 1]];
    return (long)S;
}

/* ---------------------------------------------------------------- a4 */

static void compact_row(const uint64_t *src, size_t nhaps, size_t wN, const int64_t *besthaps, size_t K,
                        uint64_t *dst, int32_t *count0) {
    int cnt1 = 0;
    if (K == nhaps) {                        /* Target.cpp:969-974: direct copy */
        size_t nopad = (nhaps + 63) / 64;
        for (size_t w = 0; w < nopad; w++) {
            uint64_t x = src[w];
            if (w == nopad - 1 && (nhaps % 64)) x &= (1ull << (nhaps % 64)) - 1;
            dst[w] = x;
            cnt1 += popc64(x);
        }
        (void)wN;
    } else {                                 /* :976-981: gather the K best haps */
        for (size_t k = 0; k < K; k++)
            if (getbit(src, (size_t)besthaps[k])) { setbit(dst, k); cnt1++; }
    }
    *count0 = (int32_t)K - cnt1;
}

void eo_cref(const uint8_t *gt, const uint64_t *sitemajor, size_t M, size_t nhaps,
             const int64_t *besthaps, size_t K, const int64_t *splits, size_t S,
             uint64_t *cref, int32_t *count0) {
    size_t wN = eo_W(nhaps), wK = eo_W(K);
    size_t Mp = 2 * S + 1;
    memset(cref, 0, Mp * wK * sizeof(uint64_t));
    uint64_t *incon = (uint64_t *)calloc(wN, sizeof(uint64_t));
    size_t nopad = (nhaps + 63) / 64;
    size_t row = 0, si = 0;
    for (size_t m = 0; m < M; m++) {
        const uint64_t *ref = sitemajor + m * wN;
        if (si < S && (size_t)splits[si] == m) {
            compact_row(incon, nhaps, wN, besthaps, K, cref + row * wK, count0 + row);
            row++;
            memset(incon, 0, wN * sizeof(uint64_t));
            compact_row(ref, nhaps, wN, besthaps, K, cref + row * wK, count0 + row);
            row++;
            si++;
        } else if (gt[m] == 0) {             /* Target.cpp:1040-1059 */
            for (size_t w = 0; w < nopad; w++) incon[w] |= ref[w];
        } else if (gt[m] == 2) {
            for (size_t w = 0; w < nopad; w++) incon[w] |= ~ref[w];
        }
    }
    compact_row(incon, nhaps, wN, besthaps, K, cref + row * wK, count0 + row);
    free(incon);
}

/* ---------------------------------------------------------------- a5 */

void eo_pbwt(const uint64_t *rows, size_t rowwords, size_t Mp, size_t K, int reverse,
             uint32_t *out, int32_t *absperm, int32_t *count0_out) {
    /* PBWT.cpp:207-285.  The prefix order starts as the identity (:212-215);
     * each row stably partitions it into the haps carrying 0, then 1; the
     * row's bits are emitted in the order BEFORE the partition, with the
     * running count of zeros after every 32 bits, and the tail word padded
     * with ones (:261-267). */
    size_t kw = 2 * ((K + 31) / 32);
    int32_t *perm = (int32_t *)malloc(K * sizeof(int32_t));
    int32_t *next = (int32_t *)malloc(K * sizeof(int32_t));
    for (size_t i = 0; i < K; i++) perm[i] = (int32_t)i;
    if (absperm) memcpy(absperm, perm, K * sizeof(int32_t));
    for (size_t midx = 0; midx < Mp; midx++) {
        size_t m = reverse ? Mp - 1 - midx : midx;
        const uint64_t *data = rows + m * rowwords;
        uint32_t *o = out + midx * kw;
        size_t cnt0 = 0;
        for (size_t i = 0; i < K; i++) cnt0 += !getbit(data, i);
        size_t p0 = 0, p1 = cnt0;
        uint32_t word = 0, mask = 1;
        for (size_t i = 0; i < K; i++) {
            int32_t h = perm[i];
            if (!getbit(data, (size_t)h)) next[p0++] = h;
            else { word |= mask; next[p1++] = h; }
            mask <<= 1;
            if (mask == 0) { *o++ = word; *o++ = (uint32_t)p0; word = 0; mask = 1; }
        }
        if (K % 32) { *o++ = word | ~(mask - 1); *o++ = (uint32_t)p0; }
        if (count0_out) count0_out[m] = (int32_t)cnt0;
        int32_t *t = perm; perm = next; next = t;
        if (absperm) memcpy(absperm + (midx + 1) * K, perm, K * sizeof(int32_t));
    }
    free(perm);
    free(next);
}

int eo_rank(const uint32_t *row, int cnt0, int from) {
    /* PBWT.cpp:367-382 */
    uint32_t off = row[2 * (from / 32) + 1];
    uint32_t field = row[2 * (from / 32)];
    uint32_t mask = 1u << (from % 32);
    uint32_t bit = field & mask;
    mask--;
    field |= mask;
    uint32_t fcnt0 = off - (uint32_t)__builtin_popcount(~field);
    if (bit) return cnt0 + (from - (int)fcnt0);
    return (int)fcnt0;
}

/* PBWT.cpp:304-365: map interval [l,r] (l>r: empty) through one row */
static void map_interval(const uint32_t *row, int cnt0, int l, int r, int *l0, int *r0, int *l1, int *r1) {
    *l0 = 0; *r0 = -1; *l1 = 0; *r1 = -1;
    if (l > r) return;
    if (l == r) {
        int i = eo_rank(row, cnt0, l);
        if (i < cnt0) { *l0 = i; *r0 = i; } else { *l1 = i; *r1 = i; }
        return;
    }
    int a0 = eo_rank(row, cnt0, l);
    int a1 = l - a0 + cnt0;
    if (a0 >= cnt0) { int t = a0; a0 = a1; a1 = t; }
    int b0 = eo_rank(row, cnt0, r);
    int b1 = r - b0 + cnt0 - 1;
    if (b0 >= cnt0) { int t = b0; b0 = b1; b1 = t; }
    *l0 = a0; *r0 = b0; *l1 = a1; *r1 = b1;
}

/* ---------------------------------------------------------------- a8 */

typedef struct {
    int left, right;          /* node indices, -1 = none */
    int l, r;                 /* interval */
    long depth;
    int errors;
} eo_node;

typedef struct {
    eo_node *nodes;
    int *freelist;
    int nfree, cap, used;
} eo_pool;

static int eo_peak_nodes = 0;
int eo_smm_peak_nodes(void) { return eo_peak_nodes; }

static int pool_new(eo_pool *p, int l, int r, long depth, int errors) {
    int i;
    if (p->nfree) i = p->freelist[--p->nfree];
    else {
        if (p->used == p->cap) {
            p->cap = p->cap ? 2 * p->cap : 1024;
            p->nodes = (eo_node *)realloc(p->nodes, p->cap * sizeof(eo_node));
            p->freelist = (int *)realloc(p->freelist, p->cap * sizeof(int));
        }
        i = p->used++;
    }
    if (p->used - p->nfree > eo_peak_nodes) eo_peak_nodes = p->used - p->nfree;
    eo_node *n = &p->nodes[i];
    n->left = n->right = -1; n->l = l; n->r = r; n->depth = depth; n->errors = errors;
    return i;
}
static void pool_del(eo_pool *p, int i) { p->freelist[p->nfree++] = i; }

typedef struct {
    const uint32_t *row; int cnt0;
    int curr_hap, missing, setmaxerrors;
    long treedepth; size_t m;
    int64_t *out; size_t nout, maxout; int overflow;
} eo_smm_ctx;

static void emit(eo_smm_ctx *c, int64_t s, int64_t e, int64_t rs, int64_t re) {
    if (c->nout >= c->maxout) { c->overflow = 1; return; }
    int64_t *o = c->out + 4 * c->nout++;
    o[0] = s; o[1] = e; o[2] = rs; o[3] = re;
}

/* TargetImp.cpp:346-435.  *lt / *rt are the parent's link slots. */
static long process_subtree(eo_pool *P, int *lt, int *rt, eo_smm_ctx *c, int perase, eo_node *scratch_matches) {
    (void)scratch_matches;
    eo_node *L = &P->nodes[*lt];
    int l0 = 0, r0 = -1, l1 = 0, r1 = -1;
    if (!perase) map_interval(c->row, c->cnt0, L->l, L->r, &l0, &r0, &l1, &r1);
    int empty0 = l0 > r0, empty1 = l1 > r1;
    int extend0 = !empty0 && (c->missing || !c->curr_hap || L->errors < c->setmaxerrors);
    int extend1 = !empty1 && (c->missing || c->curr_hap || L->errors < c->setmaxerrors);
    if (extend1) {
        int e = (c->curr_hap || c->missing) ? L->errors : L->errors + 1;
        int ni = pool_new(P, l1, r1, L->depth + 1, e);
        L = &P->nodes[*lt];
        *rt = ni;
    }
    if (extend0) {
        L->l = l0; L->r = r0; L->depth++;
        if (c->curr_hap && !c->missing) L->errors++;
    }
    if (!extend0 && !extend1) {
        if (L->depth == c->treedepth && c->treedepth > 0)
            emit(c, (int64_t)c->m - L->depth, (int64_t)c->m, L->l, L->r);
    }
    long ldepth = 0, rdepth = 0;
    int child_erase = !extend0 && !extend1;
    /* Children are visited with the slot of the matching child of the new
     * 1-node (TargetImp.cpp:383-388: "rtree ? rtree->left : rtree").  When
     * no 1-node exists the children cannot extend with 1 either (their
     * intervals are sub-intervals and their error counts are not smaller),
     * so the slot stays empty.  Slots are passed by value and written back
     * because the node pool may move while a subtree grows. */
    if (P->nodes[*lt].left >= 0) {
        int lslot = P->nodes[*lt].left;
        int rslot = (*rt >= 0) ? P->nodes[*rt].left : -1;
        ldepth = process_subtree(P, &lslot, &rslot, c, child_erase, NULL);
        P->nodes[*lt].left = lslot;
        if (*rt >= 0) P->nodes[*rt].left = rslot;
    }
    if (P->nodes[*lt].right >= 0) {
        int lslot = P->nodes[*lt].right;
        int rslot = (*rt >= 0) ? P->nodes[*rt].right : -1;
        rdepth = process_subtree(P, &lslot, &rslot, c, child_erase, NULL);
        P->nodes[*lt].right = lslot;
        if (*rt >= 0) P->nodes[*rt].right = rslot;
    }
    long depth = ldepth > rdepth ? ldepth : rdepth;
    if (extend0) {
        eo_node *N = &P->nodes[*lt];
        if (N->depth > depth) depth = N->depth;
        if (N->left >= 0 && N->right < 0 && P->nodes[N->left].l == N->l && P->nodes[N->left].r == N->r &&
            P->nodes[N->left].errors == N->errors) {
            int tmp = *lt; *lt = N->left; pool_del(P, tmp);
        } else if (N->left < 0 && N->right >= 0 && P->nodes[N->right].l == N->l && P->nodes[N->right].r == N->r &&
                   P->nodes[N->right].errors == N->errors) {
            int tmp = *lt; *lt = N->right; pool_del(P, tmp);
        }
    } else {
        pool_del(P, *lt);
        *lt = -1;
    }
    if (extend1) {
        eo_node *R = &P->nodes[*rt];
        if (R->depth > depth) depth = R->depth;
        if (R->left >= 0 && R->right < 0 && P->nodes[R->left].l == R->l && P->nodes[R->left].r == R->r &&
            P->nodes[R->left].errors == R->errors) {
            int tmp = *rt; *rt = R->left; pool_del(P, tmp);
        } else if (R->left < 0 && R->right >= 0 && P->nodes[R->right].l == R->l && P->nodes[R->right].r == R->r &&
                   P->nodes[R->right].errors == R->errors) {
            int tmp = *rt; *rt = R->right; pool_del(P, tmp);
        }
    }
    return depth;
}

long eo_smmatches(const uint32_t *refpbwt, const int32_t *count0, size_t M, size_t K,
                  const uint64_t *hap, const int64_t *miss, size_t nmiss, int setmaxerrors,
                  int64_t *out, size_t maxmatches) {
    /* TargetImp.cpp:74-246 */
    if (nmiss > M / 2) return 0;
    size_t kw = 2 * ((K + 31) / 32);
    eo_pool P = {0};
    int root = pool_new(&P, 0, (int)K - 1, 0, 0);
    size_t missidx = 0;
    size_t nextmiss = (size_t)-1;
    if (missidx < nmiss) nextmiss = (size_t)miss[missidx++];
    eo_smm_ctx c;
    memset(&c, 0, sizeof(c));
    c.setmaxerrors = setmaxerrors;
    c.out = out; c.maxout = maxmatches;
    int64_t *tmp = (int64_t *)malloc(4 * sizeof(int64_t) * (maxmatches + 1));
    long treedepth = 0;
    size_t nres = 0;
    for (size_t m = 0; m < M; m++) {
        int curr = getbit(hap, m);
        int missing = (m == nextmiss);
        if (missing) nextmiss = (missidx >= nmiss) ? (size_t)-1 : (size_t)miss[missidx++];
        int nr = pool_new(&P, 0, (int)K - 1, 0, 0);
        P.nodes[nr].left = root;
        root = nr;
        c.row = refpbwt + m * kw; c.cnt0 = count0[m];
        c.curr_hap = curr; c.missing = missing; c.treedepth = treedepth; c.m = m;
        c.out = tmp; c.nout = 0; c.maxout = maxmatches;
        int lslot = P.nodes[root].left, rslot = P.nodes[root].right;
        treedepth = process_subtree(&P, &lslot, &rslot, &c, 0, NULL);
        P.nodes[root].left = lslot; P.nodes[root].right = rslot;
        if (c.overflow) { nres = (size_t)-1; break; }
        /* TargetImp.cpp:132-136 */
        if (c.nout && (size_t)(tmp[1] - tmp[0]) >= (size_t)treedepth) {
            for (size_t i = 0; i < c.nout; i++) {
                if (nres >= maxmatches) { nres = (size_t)-1; break; }
                memcpy(out + 4 * nres, tmp + 4 * i, 4 * sizeof(int64_t));
                nres++;
            }
            if (nres == (size_t)-1) break;
        }
    }
    if (nres != (size_t)-1) {
        /* :144: process the remaining tree with erase set */
        c.row = NULL; c.cnt0 = 0; c.curr_hap = 0; c.missing = 0; c.treedepth = treedepth; c.m = M;
        c.out = tmp; c.nout = 0;
        int slot = root, rslot2 = root;
        process_subtree(&P, &slot, &rslot2, &c, 1, NULL);
        if (c.overflow) nres = (size_t)-1;
        else
            for (size_t i = 0; i < c.nout; i++) {
                if (nres >= maxmatches) { nres = (size_t)-1; break; }
                memcpy(out + 4 * nres, tmp + 4 * i, 4 * sizeof(int64_t));
                nres++;
            }
    }
    free(tmp);
    free(P.nodes);
    free(P.freelist);
    return nres == (size_t)-1 ? -1 : (long)nres;
}

/* ---------------------------------------------------------------- a9 */

void eo_impute(const int64_t *matches, size_t nmatches, const int32_t *absperm, size_t K,
               const uint64_t *sitemajor_full, size_t wN, size_t Mref, const int64_t *typed,
               size_t M, const float *af_full, size_t nrefhaps_total, const int64_t *miss,
               size_t nmiss, int imputeCalls, const uint64_t *hap, uint64_t *bits, float *dos,
               uint8_t *imputed, double *dos64) {
    /* TargetImp.cpp:474-558 (+ the constructor's initial state :28-59).
     * dos64 (optional): the FP64 dosage oracle, score/sum in double without
     * the reference's final rounding to float (-1 at uncovered sites, the
     * written value elsewhere) */
    memset(bits, 0, eo_W(Mref) * sizeof(uint64_t));
    int beforefirst = 1;
    size_t currm = 0;
    size_t mmap = (size_t)typed[0];
    size_t idx0 = 0;
    size_t missidx = 0, nextmiss = (size_t)-1;
    if (missidx < nmiss) nextmiss = (size_t)miss[missidx++];
    for (size_t mref = 0; mref < Mref; mref++) {
        if (imputed) imputed[mref] = 0;
        if (mref == mmap) {
            if (beforefirst) beforefirst = 0;
            else currm++;
            while (idx0 < nmatches && (size_t)matches[4 * idx0 + 1] <= currm) idx0++;
        }
        int missing = currm == nextmiss;
        if (missing && mref == mmap)
            nextmiss = (missidx >= nmiss) ? (size_t)-1 : (size_t)miss[missidx++];
        if (mref != mmap || missing || imputeCalls) {
            if (imputed) imputed[mref] = 1;
            if (idx0 >= nmatches || (size_t)matches[4 * idx0] > currm) {
                dos[mref] = -1.0f;                       /* DOSAGE_CONFLICT (:26) */
                if (dos64) dos64[mref] = -1.0;
            } else {
                uint64_t score = 0, sum = 0;
                float af = af_full[mref];
                float maf = af > 0.5f ? 1.0f - af : af;
                const uint64_t *row = sitemajor_full + mref * wN;
                for (size_t i = idx0; i < nmatches && (size_t)matches[4 * i] <= currm; i++) {
                    size_t st = (size_t)matches[4 * i], en = (size_t)matches[4 * i + 1];
                    size_t rs = (size_t)matches[4 * i + 2], re = (size_t)matches[4 * i + 3];
                    uint64_t single = (uint64_t)(currm - st + 1) * (uint64_t)(en - currm);
                    size_t height = re - rs + 1;
                    /* :526: float maf * size_t (as float) vs double 0.01 * size_t */
                    if ((double)(maf * (float)nrefhaps_total) < 0.01 * (double)height) {
                        sum += height * single;
                        if (af > 0.5f) score += height * single;
                    } else {
                        const int32_t *ap = absperm + en * K;
                        for (size_t r = rs; r <= re; r++) {
                            sum += single;
                            if (getbit(row, (size_t)ap[r])) score += single;
                        }
                    }
                }
                if (score > sum / 2) setbit(bits, mref);
                dos[mref] = (float)((double)score / (double)sum);
                if (dos64) dos64[mref] = (double)score / (double)sum;
            }
        } else {
            /* typed, non-missing, calls not imputed: the reference writes
             * nothing here; the restatement (like the CUDA path) writes the
             * phased allele of the typed site */
            int b = getbit(hap, currm);
            if (b) setbit(bits, mref);
            dos[mref] = b ? 1.0f : 0.0f;
            if (dos64) dos64[mref] = b ? 1.0 : 0.0;
        }
        if (mref == mmap) mmap = (currm + 1) < M ? (size_t)typed[currm + 1] : Mref;
    }
}


/* ------------------------------------------------------------------------
 * Output statistics: VCFData::writeVCFImputedBunch (VCFData.cpp:3068-3446),
 * diploid targets, in the reference's order of operations.
 * ---------------------------------------------------------------------- */
static int eo_getbit(const uint64_t *row, size_t i) { return (int)((row[i >> 6] >> (i & 63)) & 1u); }
static void eo_setbit(uint64_t *row, size_t i, int v) { if (v) row[i >> 6] |= 1ull << (i & 63); }

/* htslib's bit patterns for a missing float and the end of a shorter vector */
static float eo_bcf_float(uint32_t bits) {
    float f;
    memcpy(&f, &bits, 4);
    return f;
}
#define EO_BCF_FLOAT_MISSING 0x7F800001u
#define EO_BCF_FLOAT_VECTOR_END 0x7F800002u

long eo_site_stats(size_t ntgt, size_t mref_begin, size_t nsites, const uint64_t *bits, size_t wb,
                   const float *dos, const uint64_t *phased, size_t wM, const float *pdm, const float *pdp,
                   const uint8_t *gt, size_t M, const int32_t *typed_idx, const uint8_t *is_typed,
                   const float *af_full, const uint8_t *haploid, int overwriteCalls, int improveCalls,
                   float r2filter, float maffilter, float *ads, uint64_t *gtbits, float *ds, float *gp, float *r2o,
                   float *afo, float *mafo, int32_t *aco, int32_t *ano, uint8_t *pass, uint64_t *icnt,
                   double *itot) {
    long conflictcnt = 0;
    const float fmissing = eo_bcf_float(EO_BCF_FLOAT_MISSING), fend = eo_bcf_float(EO_BCF_FLOAT_VECTOR_END);
    for (size_t isite = 0; isite < nsites; isite++) {
        const size_t idx = mref_begin + isite;
        const float rpaf = af_full[idx];                       /* :3118 */
        const int isimputed = !is_typed[idx];
        const size_t psite = (size_t)typed_idx[idx];
        double adsum = 0.0, ad2sum = 0.0;                      /* :3119-3123 */
        int nval = 0, ac1 = 0, an = 0;
        for (size_t i = 0; i < ntgt; i++) {
            const size_t h0 = 2 * i, h1 = 2 * i + 1;
            int hap0, hap1;
            float ads0, ads1;
            const int missing = !isimputed && gt[i * M + psite] == 3;   /* :3238 */
            if (haploid && haploid[i]) {
                /* haploid target, :3192-3226 (imputed) and :3399-3437 (typed):
                 * only the first haplotype row carries the sample; the second
                 * ADS and GP2 are "vector end".  A typed, non-missing call
                 * (without --overwriteCalls) keeps the phased allele with a
                 * missing ADS and adds nothing to AF, r2, AC or AN; the
                 * reference then leaves DS and GP unset (its per-thread buffers
                 * keep an earlier site's values), and this restatement writes
                 * DS missing and GP (missing, end, end) there. */
                if (isimputed || missing || overwriteCalls) {
                    hap0 = eo_getbit(bits + h0 * wb, isite);
                    ads0 = dos[h0 * nsites + isite];
                    if (ads0 < 0) { ads0 = rpaf; hap0 = rpaf > 0.5; conflictcnt++; }
                    ads[h0 * nsites + isite] = ads0;
                    adsum += ads0;
                    ad2sum += ads0 * ads0;
                    if (ds) ds[i * nsites + isite] = ads0;
                    if (gp) {
                        double gp0 = (1.0 - ads0);
                        double gp2 = ads0;
                        gp[(3 * i) * nsites + isite] = (float)gp0;
                        gp[(3 * i + 1) * nsites + isite] = (float)gp2;
                        gp[(3 * i + 2) * nsites + isite] = fend;
                    }
                    if (hap0) ac1++;
                    an++;
                    nval++;
                } else {
                    hap0 = eo_getbit(phased + h0 * wM, psite);
                    ads[h0 * nsites + isite] = fmissing;
                    if (ds) ds[i * nsites + isite] = fmissing;
                    if (gp) {
                        gp[(3 * i) * nsites + isite] = fmissing;
                        gp[(3 * i + 1) * nsites + isite] = fend;
                        gp[(3 * i + 2) * nsites + isite] = fend;
                    }
                }
                ads[h1 * nsites + isite] = fend;
                eo_setbit(gtbits + h0 * wb, isite, hap0);
                eo_setbit(gtbits + h1 * wb, isite, 0);
                continue;
            }
            if (isimputed || missing || overwriteCalls) {      /* :3126-3152, :3246-3270 */
                hap0 = eo_getbit(bits + h0 * wb, isite);
                hap1 = eo_getbit(bits + h1 * wb, isite);
                ads0 = dos[h0 * nsites + isite];
                if (ads0 < 0) { ads0 = rpaf; hap0 = rpaf > 0.5; conflictcnt++; }
                ads1 = dos[h1 * nsites + isite];
                if (ads1 < 0) { ads1 = rpaf; hap1 = rpaf > 0.5; conflictcnt++; }
            } else {                                           /* :3272-3340 */
                hap0 = eo_getbit(phased + h0 * wM, psite);
                hap1 = eo_getbit(phased + h1 * wM, psite);
                ads0 = pdm[i * M + psite];
                ads1 = pdp[i * M + psite];
                if (improveCalls) {
                    float idos0 = dos[h0 * nsites + isite];
                    float idos1 = dos[h1 * nsites + isite];
                    float pdos0 = ads0;
                    float pdos1 = ads1;
                    if (idos0 < 0) idos0 = rpaf;
                    if (idos1 < 0) idos1 = rpaf;
                    if (idos0 > 0.5) idos0 = 1.0 - idos0;
                    if (idos1 > 0.5) idos1 = 1.0 - idos1;
                    if (pdos0 > 0.5) pdos0 = 1.0 - pdos0;
                    if (pdos1 > 0.5) pdos1 = 1.0 - pdos1;
                    float improve0 = pdos0 - idos0;
                    float improve1 = pdos1 - idos1;
                    if (improve0 + improve1 > 0) {
                        if (dos[h0 * nsites + isite] < 0) conflictcnt++;
                        if (dos[h1 * nsites + isite] < 0) conflictcnt++;
                        /* :3306-3330, the run statistics of an improved call:
                         * 0 no allele changes, 1 het->het (both change), 2
                         * hom->hom (both change), 3 het->hom, 4 hom->het (one
                         * changes); totals add the float improve0 + improve1 */
                        const int i0 = eo_getbit(bits + h0 * wb, isite), i1 = eo_getbit(bits + h1 * wb, isite);
                        int cat;
                        if (hap0 != i0 && hap1 != i1) cat = hap0 != hap1 ? 1 : 2;
                        else if (hap0 != i0 || hap1 != i1) cat = hap0 == hap1 ? 4 : 3;
                        else cat = 0;
                        if (icnt) icnt[cat]++;
                        if (itot) itot[cat] += improve0 + improve1;
                        hap0 = i0;
                        hap1 = i1;
                        ads0 = hap0 ? 1.0 - idos0 : idos0;
                        ads1 = hap1 ? 1.0 - idos1 : idos1;
                    }
                }
            }
            ads[h0 * nsites + isite] = ads0;
            ads[h1 * nsites + isite] = ads1;
            adsum += ads0 + ads1;                              /* :3154-3155 */
            ad2sum += ads0 * ads0 + ads1 * ads1;
            if (ds) ds[i * nsites + isite] = ads0 + ads1;
            if (gp) {                                          /* :3159-3166 */
                double gp0 = (1.0 - ads0) * (1.0 - ads1);
                double gp2 = ads0 * ads1;
                double gp1 = 1.0 - gp0 - gp2;
                gp[(3 * i) * nsites + isite] = (float)gp0;
                gp[(3 * i + 1) * nsites + isite] = (float)gp1;
                gp[(3 * i + 2) * nsites + isite] = (float)gp2;
            }
            if (hap0) ac1++;                                   /* :3169-3174 */
            if (hap1) ac1++;
            an += 2;
            nval += 2;
            eo_setbit(gtbits + h0 * wb, isite, hap0);
            eo_setbit(gtbits + h1 * wb, isite, hap1);
        }
        double r2 = 1.0, af = 0.0, evar = 0.0, ovar = 0.0;    /* :3363-3383 */
        if (nval) {
            af = adsum / nval;
            evar = af * (1.0 - af);
            ovar = (ad2sum - adsum * af) / nval;
            if (evar > 0.0 && ovar > 0.0) r2 = ovar / evar;
            else r2 = 0.0;
        }
        float r2f = r2;
        float aff = af;
        float maff = aff > 0.5 ? 1 - aff : aff;
        r2o[isite] = r2f;
        afo[isite] = aff;
        mafo[isite] = maff;
        aco[isite] = ac1;
        ano[isite] = an;
        pass[isite] = !(r2f < r2filter || maff < maffilter);   /* :3389 */
    }
    return conflictcnt;
}


/* ------------------------------------------------------------------------
 * Qref run-length coding of haplotype vectors: utils.h:133-191 (encode),
 * utils.h:194- (decode, here without masked samples), qref_spec.md:110-173.
 * ---------------------------------------------------------------------- */
static size_t eo_add_run(size_t len, uint8_t *dest, size_t n) {   /* utils.h:133-149 */
    while (len > 32767) {
        dest[n++] = 0xff;
        dest[n++] = 0xff;
        dest[n++] = 0;
        len -= 32767;
    }
    if (len >= 128) {
        dest[n++] = (uint8_t)((len & 0x7f) | 0x80);
        dest[n++] = (uint8_t)(len >> 7);
    } else {
        dest[n++] = (uint8_t)len;
    }
    return n;
}

long eo_rle_encode(const uint64_t *src, size_t nwords, uint8_t *enc) {
    size_t n = 0, cur = 0;
    int bit = 0;
    for (size_t i = 0; i < nwords; i++) {
        uint64_t word = bit ? ~src[i] : src[i];
        int rem = 64;
        while (rem > 0) {
            int tr = word == 0 ? rem : __builtin_ctzll(word);
            if (tr < rem) {
                cur += (size_t)tr;
                rem -= tr;
                word >>= tr;
                n = eo_add_run(cur, enc, n);
                if (n >= nwords * 8) return -1;
                cur = 0;
                bit = !bit;
                word = ~word;
            } else {
                cur += (size_t)rem;
                rem = 0;
            }
        }
    }
    if (cur) n = eo_add_run(cur, enc, n);
    if (n > nwords * 8) return -1;
    return (long)n;
}

int eo_rle_decode(const uint8_t *enc, size_t encsize, uint64_t *dest, size_t nwords) {
    size_t e = 0;
    uint64_t remlength = 0;
    int bit = 1;   /* toggled before the first run */
    for (size_t i = 0; i < nwords || e < encsize; i++) {
        uint64_t rem = 64;
        while (rem > 0) {
            while (remlength == 0) {
                if (e == encsize) {
                    if (rem % 64 == 0) {   /* ends on a word boundary: the rest is zero padding */
                        remlength = rem + (i < nwords ? (nwords - i - 1) * 64 : 0);
                        bit = 0;
                        break;
                    }
                    return -1;
                }
                remlength = enc[e] & 0x7f;
                if (enc[e] & 0x80) {
                    e++;
                    if (e == encsize) return -1;
                    remlength |= (uint64_t)enc[e] << 7;
                }
                e++;
                bit = !bit;
            }
            uint64_t fill;
            if (remlength >= rem) { fill = rem; remlength -= rem; rem = 0; }
            else { fill = remlength; rem -= remlength; remlength = 0; }
            if (bit && i < nwords) {
                uint64_t v = fill == 64 ? ~0ull : ((1ull << fill) - 1ull);
                dest[i] |= v << (64 - (rem + fill));
            }
        }
    }
    return 0;
}

int eo_qref_decode(const uint8_t *section, size_t nbytes, size_t Mref, size_t nwords, uint64_t *out) {
    size_t off = 0;
    for (size_t v = 0; v < Mref; v++) {
        uint64_t encsize;
        if (off + 8 > nbytes) return -2;
        memcpy(&encsize, section + off, 8);
        off += 8;
        uint64_t *row = out + v * nwords;
        memset(row, 0, nwords * 8);
        if (encsize) {
            if (off + encsize > nbytes) return -2;
            if (eo_rle_decode(section + off, encsize, row, nwords)) return -1;
            off += encsize;
        } else {
            if (off + nwords * 8 > nbytes) return -2;
            memcpy(row, section + off, nwords * 8);
            off += nwords * 8;
        }
    }
    return 0;
}

