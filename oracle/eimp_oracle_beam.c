/*
 * CPU restatement of EagleImp's Eagle2-style beam phasing -- TEST ORACLE.
 *
 * Test infrastructure only (see eimp_oracle.h).  Follows, function by
 * function, Target::phase / phaseExtPBWT (Target.cpp:166-777), Beam
 * (Beam.cpp:41-837), BeamPath (BeamPath.cpp:29-291), HaplotypePath
 * (HaplotypePath.cpp:36-483), BooleanHistory (BooleanHistory.cpp:31-113),
 * History (History.h:29-81) and MinMaxHeap (MinMaxHeap.h:29-214).
 *
 * Floating point follows the reference operation by operation: fp_type is
 * float (Datatypes.h:68); every place where the reference mixes in a double
 * literal or pow() is written with explicit double arithmetic and a final
 * conversion to float.  Built with -ffp-contract=off (no FMA).
 */
#include "eimp_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EO_HMAX 128

static inline int getbit(const uint64_t *v, size_t i) { return (int)((v[i >> 6] >> (i & 63)) & 1u); }
static inline void setbit(uint64_t *v, size_t i) { v[i >> 6] |= 1ull << (i & 63); }
static inline void clrbit(uint64_t *v, size_t i) { v[i >> 6] &= ~(1ull << (i & 63)); }

/* ------------------------------------------------------------ constraints */
enum { C_HOMREF = 0, C_HETKEEP = 1, C_HETSWITCH = 2, C_HOMALT = 3, C_NONE = 4 };
typedef struct { int type; int refidx; } constr_t;

/* ------------------------------------------------------------ min-max heap
 * MinMaxHeap.h:29-214, elements compared by their float key with '<'. */
typedef struct { float key; int a; int b; } hel;
typedef struct { hel *h; int n, cap; } mmheap;

static void hp_init(mmheap *q) { q->h = NULL; q->n = 0; q->cap = 0; }
static void hp_free(mmheap *q) { free(q->h); q->h = NULL; q->n = q->cap = 0; }
static inline int hp_lt(const hel *x, const hel *y) { return x->key < y->key; }
static inline void hp_swap(mmheap *q, int i, int j) { hel t = q->h[i]; q->h[i] = q->h[j]; q->h[j] = t; }
static inline unsigned long hp_log2(unsigned long x) { return x == 0 ? 0 : (unsigned long)(63 - __builtin_clzl(x)); }
static inline int hp_minlevel(int i) { return (hp_log2((unsigned long)i + 1) % 2) == 0; }
static inline int hp_parent(int i) { return (i - 1) / 2; }

static void hp_bubble_helper(mmheap *q, int i, int ismax) {
    while (1) {
        if (i == 0) return;
        int p = hp_parent(i);
        if (p == 0) return;
        int g = hp_parent(p);
        if (hp_lt(&q->h[i], &q->h[g]) ^ ismax) { hp_swap(q, g, i); i = g; }
        else return;
    }
}
static void hp_bubble(mmheap *q, int i) {
    if (i == 0) return;
    int p = hp_parent(i);
    if (hp_minlevel(i)) {
        if (hp_lt(&q->h[p], &q->h[i])) { hp_swap(q, p, i); hp_bubble_helper(q, p, 1); }
        else hp_bubble_helper(q, i, 0);
    } else {
        if (hp_lt(&q->h[i], &q->h[p])) { hp_swap(q, p, i); hp_bubble_helper(q, p, 0); }
        else hp_bubble_helper(q, i, 1);
    }
}
static void hp_trickle_helper(mmheap *q, int i, int ismax) {
    while (1) {
        int ext = i;
        int lc = 2 * i + 1;
        int n = q->n;
        if (lc < n && (hp_lt(&q->h[lc], &q->h[ext]) ^ ismax)) ext = lc;
        if (lc + 1 < n && (hp_lt(&q->h[lc + 1], &q->h[ext]) ^ ismax)) ext = lc + 1;
        int lg = 2 * lc + 1;
        for (int k = 0; k < 4 && lg + k < n; ++k)
            if (hp_lt(&q->h[lg + k], &q->h[ext]) ^ ismax) ext = lg + k;
        if (i == ext) return;
        hp_swap(q, i, ext);
        if (ext - lc > 1) {
            if (hp_lt(&q->h[hp_parent(ext)], &q->h[ext]) ^ ismax) hp_swap(q, hp_parent(ext), ext);
            i = ext;
        } else return;
    }
}
static void hp_trickle(mmheap *q, int i) { hp_trickle_helper(q, i, hp_minlevel(i) ? 0 : 1); }
static int hp_maxidx(const mmheap *q) {
    if (q->n == 1) return 0;
    if (q->n == 2) return 1;
    return hp_lt(&q->h[1], &q->h[2]) ? 2 : 1;
}
static void hp_delete(mmheap *q, int i) {
    if (i == q->n - 1) { q->n--; return; }
    hp_swap(q, i, q->n - 1);
    q->n--;
    hp_trickle(q, i);
}
static hel hp_popmin(mmheap *q) { hel e = q->h[0]; hp_delete(q, 0); return e; }
static void hp_push(mmheap *q, float key, int a, int b) {
    if (q->n == q->cap) { q->cap = q->cap ? 2 * q->cap : 64; q->h = (hel *)realloc(q->h, q->cap * sizeof(hel)); }
    q->h[q->n].key = key; q->h[q->n].a = a; q->h[q->n].b = b;
    q->n++;
    hp_bubble(q, q->n - 1);
}

/* ------------------------------------------------------------ histories */
typedef struct { uint64_t d[2]; uint64_t fill[2]; int last, histlast; } bhist;

static void bh_init(bhist *h, int H) {
    /* BooleanHistory.cpp:31-53 */
    h->histlast = H - 1;
    int lw = (H - 1) / 64;
    uint64_t mlw = (H % 64 == 0) ? 0ull : ~((1ull << (H % 64)) - 1ull);
    for (int i = 0; i < 2; i++) h->fill[i] = i < lw ? 0ull : (i == lw ? mlw : ~0ull);
    h->last = -1;
    h->d[0] = h->fill[0]; h->d[1] = h->fill[1];
}
static void bh_push(bhist *h, int b) {
    /* BooleanHistory.cpp:55-70 */
    uint64_t carry = b ? 1ull : 0ull;
    for (int i = 0; i < 2; i++) {
        uint64_t nc = h->d[i] >> 63;
        h->d[i] = (h->d[i] << 1) | carry;
        carry = nc;
    }
    if (h->last != h->histlast) h->last++;
    h->d[0] |= h->fill[0]; h->d[1] |= h->fill[1];
}
static inline int bh_at(const bhist *h, int pos) { return (int)((h->d[pos / 64] >> (pos % 64)) & 1ull); }
static int bh_numequal(const bhist *a, const bhist *b) {
    /* BooleanHistory.cpp:99-113 */
    uint64_t t = a->d[0] ^ b->d[0];
    if (t) return __builtin_ctzll(t);
    t = a->d[1] ^ b->d[1];
    if (t) return 64 + __builtin_ctzll(t);
    return 128;
}
static int bh_equal(const bhist *a, const bhist *b) {
    /* BooleanHistory.cpp:91-97: the loop compares a third 8-byte slot after
     * the two data words, i.e. the members 'last' and 'histlast' */
    return a->d[0] == b->d[0] && a->d[1] == b->d[1] && a->last == b->last && a->histlast == b->histlast;
}

/* ------------------------------------------------------------ PBWT view */
typedef struct {
    const uint32_t *rows;   /* fwd rows then bck rows, kw words each */
    const int32_t *count0;  /* per natural row index */
    int Mp, K, kw, reverse;
    float Kinv;
} pbwt_v;

static inline int rank_(const uint32_t *row, int cnt0, int from) { return eo_rank(row, cnt0, from); }

static void pv_map(const pbwt_v *pv, int m, int l, int r, int *l0, int *r0, int *l1, int *r1) {
    /* PBWT.cpp:288-365 */
    const uint32_t *row = pv->rows + (size_t)(pv->reverse ? (2 * pv->Mp - 1 - m) : m) * pv->kw;
    int cnt0 = pv->count0[m];
    *l0 = 0; *r0 = -1; *l1 = 0; *r1 = -1;
    if (l > r) return;
    if (l == r) {
        int i = rank_(row, cnt0, l);
        if (i < cnt0) { *l0 = i; *r0 = i; } else { *l1 = i; *r1 = i; }
        return;
    }
    int a0 = rank_(row, cnt0, l);
    int a1 = l - a0 + cnt0;
    if (a0 >= cnt0) { int t = a0; a0 = a1; a1 = t; }
    int b0 = rank_(row, cnt0, r);
    int b1 = r - b0 + cnt0 - 1;
    if (b0 >= cnt0) { int t = b0; b0 = b1; b1 = t; }
    *l0 = a0; *r0 = b0; *l1 = a1; *r1 = b1;
}

/* ------------------------------------------------------------ haplotype paths */
typedef struct { int l, r; } ivl;

typedef struct {
    bhist path;
    float p; int scaleexp;                /* HaplotypePathProbability prob */
    float ph[EO_HMAX]; int phstart, phsize; /* History<fp_type> probHist */
    ivl *iv; int niv;                     /* pbwtInt */
    ivl *ext[2]; int next[2];             /* extensionPbwtInt */
    float extp[2]; int extscaleexp;
    int active[2], toextend[2], refcnt[2];
} hpath;

static inline float *ph_at(hpath *h, int pos) { return &h->ph[(pos + h->phstart) & (h->phsize - 1)]; }
static inline void ph_push(hpath *h, float v) { h->phstart = (h->phstart - 1) & (h->phsize - 1); h->ph[h->phstart] = v; }

typedef struct {
    int mat, pat;
    float prob, weight;
    float pErr; int nErr; float pErrPath, pErrPathp1;
    float extp[4]; int active[4]; int actidx;
    int extgeno;
    int prev, next;
} bpath;

typedef struct {
    int H, P, Delta;
    float pErr, pLimit, expectIBDcM;
    const float *cmd; int ncmd;
    const int64_t *calls; int ncalls;
    const uint8_t *tgt;         /* condensed genotypes at split sites */
    const constr_t *constr; int S;
    int reverse;
    int cursor, curridx, refidx;
    pbwt_v pv;
    /* beam list */
    bpath *bp; int bpcap, head, tail, nbp; int *bpfree; int nbpfree;
    /* happaths */
    hpath *hp; int hpcap; int *hpfree; int nhpfree;
    int *happaths; int nhap, happcap;
    float prec[EO_HMAX];
    int error;
} beam_t;

static int hp_alloc(beam_t *B) {
    if (B->nhpfree) return B->hpfree[--B->nhpfree];
    if (B->hpcap % 256 == 0) {
        int ncap = B->hpcap + 256;
        B->hp = (hpath *)realloc(B->hp, ncap * sizeof(hpath));
        B->hpfree = (int *)realloc(B->hpfree, ncap * sizeof(int));
        for (int i = B->hpcap; i < ncap; i++) {
            B->hp[i].iv = (ivl *)malloc(B->H * sizeof(ivl));
            B->hp[i].ext[0] = (ivl *)malloc(B->H * sizeof(ivl));
            B->hp[i].ext[1] = (ivl *)malloc(B->H * sizeof(ivl));
        }
    }
    return B->hpcap++;
}
static void hp_release(beam_t *B, int i) { B->hpfree[B->nhpfree++] = i; }

static int bp_alloc(beam_t *B) {
    if (B->nbpfree) return B->bpfree[--B->nbpfree];
    static const int CH = 256;
    if (B->bpcap % CH == 0) {
        B->bp = (bpath *)realloc(B->bp, (B->bpcap + CH) * sizeof(bpath));
        B->bpfree = (int *)realloc(B->bpfree, (B->bpcap + CH) * sizeof(int));
    }
    return B->bpcap++;
}
static void list_push_back(beam_t *B, int i) {
    B->bp[i].next = -1; B->bp[i].prev = B->tail;
    if (B->tail >= 0) B->bp[B->tail].next = i; else B->head = i;
    B->tail = i; B->nbp++;
}
static int list_erase(beam_t *B, int i) {
    int n = B->bp[i].next, p = B->bp[i].prev;
    if (p >= 0) B->bp[p].next = n; else B->head = n;
    if (n >= 0) B->bp[n].prev = p; else B->tail = p;
    B->bpfree[B->nbpfree++] = i; B->nbp--;
    return n;
}
static void happ_push(beam_t *B, int id) {
    if (B->nhap == B->happcap) { B->happcap = B->happcap ? 2 * B->happcap : 64; B->happaths = (int *)realloc(B->happaths, B->happcap * sizeof(int)); }
    B->happaths[B->nhap++] = id;
}

/* HaplotypePath.cpp:36-53 */
static int hpath_new(beam_t *B, int alt) {
    int id = hp_alloc(B);
    hpath *h = &B->hp[id];
    bh_init(&h->path, B->H);
    bh_push(&h->path, alt);
    h->p = 1.0f; h->scaleexp = 0;
    int l2 = 63 - __builtin_clzll((unsigned long long)B->H);
    if ((1 << l2) != B->H) l2++;
    h->phsize = 1 << l2;
    memset(h->ph, 0, sizeof(h->ph));
    h->phstart = 0;
    ph_push(h, 1.0f);
    h->niv = 0; h->next[0] = h->next[1] = 0;
    h->extp[0] = h->extp[1] = 0.0f; h->extscaleexp = 0;
    h->active[0] = h->active[1] = 0; h->toextend[0] = h->toextend[1] = 0; h->refcnt[0] = h->refcnt[1] = 0;
    return id;
}

/* HaplotypePath.cpp:55-75: copy of 'other' with extension e applied */
static int hpath_copy_ext(beam_t *B, int oid, int e) {
    int id = hp_alloc(B);
    hpath *h = &B->hp[id], *o = &B->hp[oid];
    ivl *iv = h->iv, *e0 = h->ext[0], *e1 = h->ext[1];
    h->path = o->path;
    h->p = o->extp[e]; h->scaleexp = o->extscaleexp;
    memcpy(h->ph, o->ph, sizeof(h->ph)); h->phstart = o->phstart; h->phsize = o->phsize;
    h->iv = iv; h->ext[0] = e0; h->ext[1] = e1;
    memcpy(h->iv, o->ext[e], o->next[e] * sizeof(ivl)); h->niv = o->next[e];
    h->next[0] = h->next[1] = 0;
    h->active[0] = h->active[1] = 0; h->toextend[0] = h->toextend[1] = 0; h->refcnt[0] = h->refcnt[1] = 0;
    bh_push(&h->path, e);
    ph_push(h, o->extp[e]);
    h->extp[0] = h->extp[1] = 0.0f; h->extscaleexp = 0;
    return id;
}

/* HaplotypePath.cpp:77-103 */
static void hpath_apply(hpath *h, int e) {
    bh_push(&h->path, e);
    h->p = h->extp[e]; h->scaleexp = h->extscaleexp;
    ph_push(h, h->extp[e]);
    ivl *t = h->iv; h->iv = h->ext[e]; h->ext[e] = t; h->niv = h->next[e]; h->next[e] = 0;
    h->extp[0] = h->extp[1] = 0.0f; h->extscaleexp = 0;
    h->active[0] = h->active[1] = 0; h->toextend[0] = h->toextend[1] = 0; h->refcnt[0] = h->refcnt[1] = 0;
}

static void hpath_mark_deleted(hpath *h, int e) {   /* :105-109 */
    h->refcnt[e]--;
    if (h->refcnt[e] == 0) h->active[e] = 0;
}

static void hpath_mark_required(hpath *h, const constr_t *c) {  /* :139-158 */
    if (c->type == C_NONE) { h->toextend[0] = 1; h->toextend[1] = 1; return; }
    int hb = bh_at(&h->path, c->refidx);
    if ((c->type == C_HETKEEP && hb == 0) || (c->type == C_HETSWITCH && hb == 1) || c->type == C_HOMREF)
        h->toextend[0] = 1;
    else if ((c->type == C_HETKEEP && hb == 1) || (c->type == C_HETSWITCH && hb == 0) || c->type == C_HOMALT)
        h->toextend[1] = 1;
}

/* HaplotypePath.cpp:224-258 */
static void hpath_update_scaling(hpath *h) {
    int e = ilogbf(h->p);
    int ns = h->scaleexp;
    if (abs(e) >= 20) {
        ns += e;
        double f = pow(2.0, (double)(-e));
        for (int i = 0; i <= h->niv; i++) { float *x = ph_at(h, i); *x = (float)((double)*x * f); }
    }
    h->extscaleexp = ns;
}

/* HaplotypePath.cpp:260-479 */
static void hpath_calc(beam_t *B, hpath *h, const hpath *prev, int cursor, int copy, float *p0o, float *p1o) {
    const pbwt_v *pv = &B->pv;
    int H = B->H;
    int calc0 = h->toextend[0], calc1 = h->toextend[1];
    float p0 = 0.0f, p1 = 0.0f;
    float tmp[EO_HMAX];
    int lim = H < h->niv + 1 ? H : h->niv + 1;
    for (int i = 0; i < lim; i++) tmp[i] = *ph_at(h, i) * B->prec[i];
    ivl *e0 = h->ext[0], *e1 = h->ext[1];
    int n0 = 0, n1 = 0;
    int cnt0 = pv->count0[2 * cursor + 1];
    if (cnt0 > 0) {
        if (calc0) p0 = (float)cnt0 * tmp[0];
        e0[n0].l = 0; e0[n0].r = cnt0 - 1; n0++;
    }
    if (cnt0 < pv->K) {
        if (calc1) p1 = (float)(pv->K - cnt0) * tmp[0];
        e1[n1].l = cnt0; e1[n1].r = pv->K - 1; n1++;
    }
    int bothempty = 0;
    int i = 1;
    int lc = copy < h->niv + 1 ? copy : h->niv + 1;
    for (; !bothempty && i < lc; i++) {
        bothempty = 1;
        if (prev->next[0] > i) {
            ivl t = prev->ext[0][i];
            if (calc0) p0 += (float)(t.r - t.l + 1) * tmp[i];
            e0[n0++] = t;
            bothempty = 0;
        }
        if (prev->next[1] > i) {
            ivl t = prev->ext[1][i];
            if (calc1) p1 += (float)(t.r - t.l + 1) * tmp[i];
            e1[n1++] = t;
            bothempty = 0;
        }
    }
    for (; !bothempty && i < lim; i++) {
        ivl from = h->iv[i - 1];
        int t0l = 0, t0r = -1, t1l = 0, t1r = -1;
        if (i > 1 && h->iv[i - 2].l == from.l && h->iv[i - 2].r == from.r) {
            if (n0 == i) { t0l = e0[n0 - 1].l; t0r = e0[n0 - 1].r; }
            if (n1 == i) { t1l = e1[n1 - 1].l; t1r = e1[n1 - 1].r; }
        } else {
            int cl, cr, il, ir;
            pv_map(pv, pv->reverse ? 2 * (cursor + 1) : 2 * cursor, from.l, from.r, &cl, &cr, &il, &ir);
            pv_map(pv, 2 * cursor + 1, cl, cr, &t0l, &t0r, &t1l, &t1r);
        }
        bothempty = 1;
        if (t0l <= t0r) {
            if (calc0) p0 += (float)(t0r - t0l + 1) * tmp[i];
            e0[n0].l = t0l; e0[n0].r = t0r; n0++;
            bothempty = 0;
        }
        if (t1l <= t1r) {
            if (calc1) p1 += (float)(t1r - t1l + 1) * tmp[i];
            e1[n1].l = t1l; e1[n1].r = t1r; n1++;
            bothempty = 0;
        }
    }
    h->next[0] = n0; h->next[1] = n1;
    *p0o = p0; *p1o = p1;
}

/* HaplotypePath.cpp:162-222 */
static int hpath_extend(beam_t *B, int id, int previd, int cursor) {
    hpath *h = &B->hp[id];
    hpath_update_scaling(h);
    int copy = 0;
    const hpath *prev = NULL;
    if (previd >= 0) {
        prev = &B->hp[previd];
        int ne = bh_numequal(&h->path, &prev->path);
        copy = B->H < 1 + ne ? B->H : 1 + ne;
    }
    float p0, p1;
    hpath_calc(B, h, prev, cursor, copy, &p0, &p1);
    h->extp[0] = p0; h->extp[1] = p1;
    h->active[0] = h->toextend[0]; h->active[1] = h->toextend[1];
    return h->extscaleexp;
}

/* ------------------------------------------------------------ beam paths */
static int incon_(int ext, int g) {   /* BeamPath.cpp:246-274 */
    switch (g) {
    case 1: return ext == 0 || ext == 3;
    case 0: return ext > 0;
    case 2: return ext < 3;
    default: return 1;
    }
}

static void bp_update_errors(bpath *b, int ext, int delerr) {   /* BeamPath.cpp:209-228 */
    int add = (incon_(ext, b->extgeno) ? 1 : 0) - (delerr ? 1 : 0);
    b->nErr += add;
    if (add < 0) { b->pErrPathp1 = b->pErrPath; b->pErrPath = b->pErrPath / b->pErr; }
    else for (int a = 0; a < add; a++) { b->pErrPath = b->pErrPathp1; b->pErrPathp1 = b->pErrPathp1 * b->pErr; }
}

static void bp_update_actidx(bpath *b) {
    b->actidx = -1;
    for (int i = 3; i >= 0; i--) if (b->active[i]) { b->actidx = i; break; }
}
static int bp_next_active(const bpath *b, int x) {
    for (int i = x - 1; i >= 0; i--) if (b->active[i]) return i;
    return -1;
}

static void bp_mark_deleted(beam_t *B, bpath *b, int ext) {   /* BeamPath.cpp:101-112 */
    b->active[ext] = 0;
    hpath_mark_deleted(&B->hp[B->happaths[b->mat]], ext / 2);
    hpath_mark_deleted(&B->hp[B->happaths[b->pat]], ext % 2);
    bp_update_actidx(b);
}

static inline void bp_single(bpath *b, int id, float p1, float p2, float scale, int incon, float *maxP) {
    b->extp[id] = p1 * p2 * scale;
    if (incon) b->extp[id] = b->extp[id] * b->pErrPathp1;
    else b->extp[id] = b->extp[id] * b->pErrPath;
    if (*maxP < b->extp[id]) *maxP = b->extp[id];
    b->active[id] = 1;
    b->actidx = id;
}

/* BeamPath.cpp:121-197 */
static float bp_extend(beam_t *B, bpath *b, int g, const constr_t *c, int bpscaleexp) {
    b->extgeno = g;
    hpath *pm = &B->hp[B->happaths[b->mat]], *pp = &B->hp[B->happaths[b->pat]];
    float pm0 = pm->extp[0], pm1 = pm->extp[1], pp0 = pp->extp[0], pp1 = pp->extp[1];
    int c0 = pm->active[0], c1 = pm->active[1], d0 = pp->active[0], d1 = pp->active[1];
    float scale = (float)pow(2.0, (double)(pm->extscaleexp + pp->extscaleexp + bpscaleexp));
    float maxP = 0.0f;
    int t = c->type;
    int hb = (t == C_HETKEEP || t == C_HETSWITCH) ? bh_at(&pm->path, c->refidx) : 0;
    if (t == C_NONE || t == C_HOMREF) {
        if (c0 && d0) { bp_single(b, 0, pm0, pp0, scale, incon_(0, g), &maxP); pm->refcnt[0]++; pp->refcnt[0]++; }
    }
    if (t == C_NONE || (t == C_HETKEEP && hb == 0) || (t == C_HETSWITCH && hb == 1)) {
        if (c0 && d1) { bp_single(b, 1, pm0, pp1, scale, incon_(1, g), &maxP); pm->refcnt[0]++; pp->refcnt[1]++; }
    }
    if (t == C_NONE || (t == C_HETKEEP && hb == 1) || (t == C_HETSWITCH && hb == 0)) {
        if (c1 && d0) { bp_single(b, 2, pm1, pp0, scale, incon_(2, g), &maxP); pm->refcnt[1]++; pp->refcnt[0]++; }
    }
    if (t == C_NONE || t == C_HOMALT) {
        if (c1 && d1) { bp_single(b, 3, pm1, pp1, scale, incon_(3, g), &maxP); pm->refcnt[1]++; pp->refcnt[1]++; }
    }
    return maxP;
}

/* ------------------------------------------------------------ beam */
static void beam_calc_rec(beam_t *B) {   /* Beam.cpp:541-573 */
    int c = B->reverse ? B->cursor + 1 : B->cursor;
    float cursordiff = B->reverse ? B->cmd[B->cursor] : B->cmd[B->cursor + 1];
    float cd = 0.0f;
    for (int i = 0; i < B->H; i++) {
        float tmp1 = (float)(1.0 + (double)(cd / B->expectIBDcM));
        float pr = (float)(1.0 / (double)(tmp1 * tmp1));
        float tmp2 = (float)(1.0 + (double)((cd + cursordiff) / B->expectIBDcM));
        pr = (float)((double)pr - 1.0 / (double)(tmp2 * tmp2));
        pr = fmaxf(fminf(pr, 1.0f), 0.000001f);
        B->prec[i] = pr * B->pv.Kinv;
        cd = cd + B->cmd[c];
        if (B->reverse) { c++; if (c >= B->ncmd) break; }
        else { if (c == 0) break; c--; }
    }
}

static void beam_init(beam_t *B) {   /* Beam.cpp:41-92 */
    B->cursor = B->reverse ? B->S : -1;
    B->curridx = -1; B->refidx = -1;
    for (int i = 0; i < EO_HMAX; i++) B->prec[i] = 0.0f;
    int mat = hpath_new(B, 0), pat = hpath_new(B, 1);
    B->nhap = 0;
    happ_push(B, mat); happ_push(B, pat);
    int b = bp_alloc(B);
    bpath *x = &B->bp[b];
    hpath *hm = &B->hp[mat], *hq = &B->hp[pat];
    x->mat = 0; x->pat = 1; x->weight = 1.0f;
    x->pErr = B->pErr; x->nErr = 0; x->pErrPath = 1.0f; x->pErrPathp1 = 1.0f * B->pErr;
    x->prob = (float)(pow(2.0, (double)(hm->scaleexp + hq->scaleexp)) * (double)hm->p * (double)hq->p * 1.0);
    for (int i = 0; i < 4; i++) { x->extp[i] = 0.0f; x->active[i] = 0; }
    x->actidx = -1; x->extgeno = 3;
    B->head = B->tail = -1; B->nbp = 0;
    list_push_back(B, b);
}

static int beam_prune(beam_t *B, float maxP, const constr_t *c) {   /* Beam.cpp:577-787 */
    float limit = B->pLimit * maxP;
    mmheap q; hp_init(&q);
    for (int it = B->head; it >= 0; it = B->bp[it].next) {
        bpath *b = &B->bp[it];
        int ex = b->actidx;
        while (ex >= 0) {
            float p = b->extp[ex];
            if (p >= limit) {
                if (q.n < B->P || (q.n == B->P && p > q.h[0].key)) {
                    if (q.n == B->P) {
                        hel e = hp_popmin(&q);
                        bp_mark_deleted(B, &B->bp[e.a], e.b);
                    }
                    hp_push(&q, p, it, ex);
                } else bp_mark_deleted(B, b, ex);
            } else bp_mark_deleted(B, b, ex);
            ex = c->type == C_NONE ? ex - 1 : -1;
        }
    }
    if (q.n == 0) { hp_free(&q); return 0; }
    int wse = -ilogbf(B->bp[q.h[0].a].weight);
    int delerr = B->bp[q.h[hp_maxidx(&q)].a].nErr > 0;
    hp_free(&q);

    /* apply haplotype path extensions (:684-726) */
    int nold = B->nhap;
    int *old = (int *)malloc((nold ? nold : 1) * sizeof(int));
    memcpy(old, B->happaths, nold * sizeof(int));
    int next0 = 0;
    for (int i = 0; i < nold; i++) if (B->hp[old[i]].active[0]) next0++;
    int *mapz = (int *)malloc((nold ? nold : 1) * sizeof(int));
    int *mapo = (int *)malloc((nold ? nold : 1) * sizeof(int));
    B->nhap = next0;
    int one = next0, zero = 0;
    for (int i = 0; i < nold; i++) {
        int id = old[i];
        hpath *h = &B->hp[id];
        mapz[i] = zero; mapo[i] = one;
        if (!(h->active[0] || h->active[1])) { hp_release(B, id); continue; }
        if (h->active[0] && h->active[1]) {
            int cp = hpath_copy_ext(B, id, 1);
            happ_push(B, cp); one++;
            hpath_apply(&B->hp[id], 0);
            B->happaths[zero++] = id;
            continue;
        }
        if (h->active[0]) { hpath_apply(h, 0); B->happaths[zero++] = id; }
        else { hpath_apply(h, 1); happ_push(B, id); one++; }
    }

    /* apply beam path extensions (:736-779) */
    int last = B->tail;
    int it = B->head;
    while (1) {
        bpath *b = &B->bp[it];
        int ex = b->actidx;
        if (ex >= 0) {
            int mat[2] = {mapz[b->mat], mapo[b->mat]};
            int pat[2] = {mapz[b->pat], mapo[b->pat]};
            int nx = bp_next_active(b, ex);
            while (nx != -1) {
                int ni = bp_alloc(B);
                b = &B->bp[it];
                bpath *n = &B->bp[ni];
                /* BeamPath.cpp:44-68 */
                n->mat = mat[ex / 2]; n->pat = pat[ex % 2];
                n->prob = b->extp[ex]; n->weight = b->weight;
                n->pErr = b->pErr; n->nErr = b->nErr; n->pErrPath = b->pErrPath; n->pErrPathp1 = b->pErrPathp1;
                for (int k = 0; k < 4; k++) n->active[k] = 0;
                n->actidx = -1; n->extgeno = b->extgeno;
                if (wse != 0) n->weight = (float)((double)n->weight * pow(2.0, (double)wse));
                bp_update_errors(n, ex, delerr);
                for (int k = 0; k < 4; k++) n->extp[k] = 0.0f;
                n->extgeno = 3;
                list_push_back(B, ni);
                ex = nx;
                nx = bp_next_active(b, nx);
            }
            /* BeamPath.cpp:70-96 */
            b->mat = mat[ex / 2]; b->pat = pat[ex % 2];
            b->prob = b->extp[ex];
            if (wse != 0) b->weight = (float)((double)b->weight * pow(2.0, (double)wse));
            bp_update_errors(b, ex, delerr);
            for (int k = 0; k < 4; k++) { b->extp[k] = 0.0f; b->active[k] = 0; }
            b->actidx = -1; b->extgeno = 3;
            if (it == last) break;
            it = B->bp[it].next;
        } else {
            if (it == last) { list_erase(B, it); break; }
            it = list_erase(B, it);
        }
    }
    free(old); free(mapz); free(mapo);
    return 1;
}

static void beam_merge(beam_t *B) {   /* Beam.cpp:790-837 */
    int n = B->nhap;
    /* key (k0,k1) -> beam path index; k0 <= k1 < n */
    int *map = (int *)malloc((size_t)n * n * sizeof(int));
    for (int i = 0; i < n * n; i++) map[i] = -1;
    int it = B->head;
    while (it >= 0) {
        bpath *b = &B->bp[it];
        int mr = b->mat;
        while (mr > 0 && bh_equal(&B->hp[B->happaths[mr]].path, &B->hp[B->happaths[mr - 1]].path)) mr--;
        int pr = b->pat;
        while (pr > 0 && bh_equal(&B->hp[B->happaths[pr]].path, &B->hp[B->happaths[pr - 1]].path)) pr--;
        int k0 = mr, k1 = pr;
        if (k0 > k1) { k0 = pr; k1 = mr; }
        int key = k0 * n + k1;
        int m = map[key];
        if (m >= 0) {
            bpath *o = &B->bp[m];
            if (o->prob > b->prob) {
                o->weight = o->weight + b->weight * (b->prob / o->prob);
                it = list_erase(B, it);
            } else {
                b->weight = b->weight + o->weight * (o->prob / b->prob);
                list_erase(B, m);
                map[key] = it;
                it = B->bp[it].next;
            }
        } else {
            map[key] = it;
            it = b->next;
        }
    }
    free(map);
}

static int beam_advance(beam_t *B) {   /* Beam.cpp:263-539 */
    B->cursor += B->reverse ? -1 : 1;
    int bpscaleexp = 0;
    beam_calc_rec(B);
    constr_t c = B->constr[B->cursor];
    int repeat;
    do {
        float maxP = 0.0f;
        for (int it = B->head; it >= 0; it = B->bp[it].next) {
            bpath *b = &B->bp[it];
            hpath_mark_required(&B->hp[B->happaths[b->mat]], &c);
            hpath_mark_required(&B->hp[B->happaths[b->pat]], &c);
        }
        int prev = -1;
        int minse = 0, maxse = INT_MIN;
        for (int i = 0; i < B->nhap; i++) {
            int id = B->happaths[i];
            hpath *h = &B->hp[id];
            if (h->toextend[0] || h->toextend[1]) {
                int se = hpath_extend(B, id, prev, B->cursor);
                prev = id;
                if (se < minse) minse = se;
                if (se > maxse) maxse = se;
            }
        }
        bpscaleexp = -(maxse + minse);
        for (int it = B->head; it >= 0; it = B->bp[it].next) {
            float mp = bp_extend(B, &B->bp[it], B->tgt[B->cursor], &c, bpscaleexp);
            if (maxP < mp) maxP = mp;
        }
        if (beam_prune(B, maxP, &c)) repeat = 0;
        else {
            if (c.type != C_NONE) { c.type = C_NONE; repeat = 1; }
            else { B->error = 1; return -1; }
        }
    } while (repeat);
    beam_merge(B);
    return 0;
}

static float beam_call_keep(beam_t *B, int ci, int twoback) {   /* Beam.cpp:95-185 */
    int front = B->reverse ? (int)(B->calls[ci] - B->Delta > 0 ? B->calls[ci] - B->Delta : 0)
                           : (int)(B->calls[ci] + B->Delta < B->S - 1 ? B->calls[ci] + B->Delta : B->S - 1);
    B->curridx = B->reverse ? (int)B->calls[ci] - front : front - (int)B->calls[ci];
    int r = B->reverse ? (int)(twoback ? B->calls[ci + 2] : B->calls[ci + 1])
                       : (int)(twoback ? B->calls[ci - 2] : B->calls[ci - 1]);
    B->refidx = B->reverse ? r - front : front - r;
    while ((B->reverse && B->cursor > front) || (!B->reverse && B->cursor < front))
        if (beam_advance(B)) return -1.0f;
    float acckp = 0.0f, accsp = 0.0f;
    for (int it = B->head; it >= 0; it = B->bp[it].next) {
        bpath *b = &B->bp[it];
        const hpath *hm = &B->hp[B->happaths[b->mat]], *hq = &B->hp[B->happaths[b->pat]];
        int cf = bh_at(&hm->path, B->curridx), cs = bh_at(&hq->path, B->curridx);
        int rf = bh_at(&hm->path, B->refidx), rs = bh_at(&hq->path, B->refidx);
        float p = b->weight * b->prob;
        if (cf != cs && rf != rs) {
            if (cf == rf) acckp = acckp + p; else accsp = accsp + p;
        } else {
            acckp = acckp + p / 2.0f;
            accsp = accsp + p / 2.0f;
        }
    }
    float ret = 0.5f;
    if (acckp + accsp > 0.0f) ret = acckp / (acckp + accsp);
    return ret;
}

static float beam_call_dosage(beam_t *B, int si) {   /* Beam.cpp:187-261 */
    int front = B->reverse ? (si - B->Delta > 0 ? si - B->Delta : 0)
                           : (si + B->Delta < B->S - 1 ? si + B->Delta : B->S - 1);
    B->curridx = B->reverse ? si - front : front - si;
    B->refidx = -1;
    while ((B->reverse && B->cursor > front) || (!B->reverse && B->cursor < front))
        if (beam_advance(B)) return -1.0f;
    float dos = 0.0f, ptot = 0.0f;
    for (int it = B->head; it >= 0; it = B->bp[it].next) {
        bpath *b = &B->bp[it];
        const hpath *hm = &B->hp[B->happaths[b->mat]], *hq = &B->hp[B->happaths[b->pat]];
        int cf = bh_at(&hm->path, B->curridx), cs = bh_at(&hq->path, B->curridx);
        float p = b->weight * b->prob;
        ptot = ptot + p;
        if (cf == cs) { if (cf == 1) dos = dos + 2.0f * p; }
        else dos = dos + p;
    }
    float ret = 1.0f;
    if (ptot > 0.0f) ret = dos / ptot;
    return ret;
}

static void beam_setup(beam_t *B, int H, int P, int Delta, const eo_phase_params *p, const float *cmd, int S,
                       const int64_t *calls, int ncalls, const uint8_t *tgt, const constr_t *constr,
                       const pbwt_v *pv, int reverse) {
    memset(B, 0, sizeof(*B));
    B->H = H; B->P = P; B->Delta = Delta;
    B->pErr = p->pErr; B->pLimit = p->pLimit; B->expectIBDcM = p->expectIBDcM;
    B->cmd = cmd; B->ncmd = S + 1; B->calls = calls; B->ncalls = ncalls; B->tgt = tgt;
    B->constr = constr; B->S = S; B->pv = *pv; B->pv.reverse = reverse; B->reverse = reverse;
    B->head = B->tail = -1;
    beam_init(B);
}

static void beam_free(beam_t *B) {
    for (int i = 0; i < B->hpcap; i++) { free(B->hp[i].iv); free(B->hp[i].ext[0]); free(B->hp[i].ext[1]); }
    free(B->hp); free(B->hpfree); free(B->bp); free(B->bpfree); free(B->happaths);
}

/* ------------------------------------------------------------ target */
static size_t hist_len(int hsize, float hist) {
    /* Target.cpp:326,466: static_cast<size_t>((HistorySize * hist) + 0.5) */
    return (size_t)((double)((float)hsize * hist) + 0.5);
}

int eo_phase(const uint8_t *gt, const uint64_t *hapmajor, const uint64_t *sitemajor,
             const float *cm, size_t M, size_t nhaps, const eo_phase_params *p,
             uint64_t *mat, uint64_t *pat, float *dos_mat, float *dos_pat,
             float *totalconf, size_t *ncallsites) {
    size_t wM = eo_W(M), K = (size_t)p->K;
    if (K > nhaps) K = nhaps;
    memset(mat, 0, wM * sizeof(uint64_t));
    memset(pat, 0, wM * sizeof(uint64_t));
    for (size_t m = 0; m < M; m++) { dos_mat[m] = 0.0f; dos_pat[m] = 0.0f; }
    *totalconf = 0.0f; *ncallsites = 0;

    /* prepPhase (Target.cpp:95-163) */
    uint64_t *gtw = (uint64_t *)calloc(2 * wM, sizeof(uint64_t));
    for (size_t m = 0; m < M; m++) {
        if (gt[m] == 0 || gt[m] == 3) gtw[2 * (m / 64)] |= 1ull << (m % 64);
        if (gt[m] == 2 || gt[m] == 3) gtw[2 * (m / 64) + 1] |= 1ull << (m % 64);
    }
    int64_t *bh = (int64_t *)malloc(K * sizeof(int64_t));
    eo_besthaps(gtw, hapmajor, nhaps, wM, K, bh, NULL);
    uint64_t *monos = (uint64_t *)malloc(wM * sizeof(uint64_t));
    eo_monos(hapmajor, wM, M, bh, K, monos);
    int64_t *splits = (int64_t *)malloc((M + 1) * sizeof(int64_t));
    int64_t *calls = (int64_t *)malloc((M + 1) * sizeof(int64_t));
    float *cmd = (float *)malloc((M + 2) * sizeof(float));
    size_t ncalls = 0;
    long S = eo_calllocs(gt, monos, cm, M, p->cMmaxsplit, splits, calls, &ncalls, cmd);
    if (S == 0) ncalls = 0;

    /* condensed reference + PBWT (Target.cpp:250-282) */
    size_t Mp = 2 * (size_t)S + 1, wK = eo_W(K), kw = 2 * ((K + 31) / 32);
    uint64_t *cref = (uint64_t *)malloc(Mp * wK * sizeof(uint64_t));
    int32_t *count0 = (int32_t *)malloc(Mp * sizeof(int32_t));
    eo_cref(gt, sitemajor, M, nhaps, bh, K, splits, (size_t)S, cref, count0);
    uint32_t *pb = (uint32_t *)malloc(2 * Mp * kw * sizeof(uint32_t));
    eo_pbwt(cref, wK, Mp, K, 0, pb, NULL, NULL);
    eo_pbwt(cref, wK, Mp, K, 1, pb + Mp * kw, NULL, NULL);
    pbwt_v pv = {pb, count0, (int)Mp, (int)K, (int)kw, 0, (float)(1.0 / (double)(float)K)};

    uint8_t *tg = (uint8_t *)malloc((size_t)S + 1);
    for (long s = 0; s < S; s++) tg[s] = gt[splits[s]];
    constr_t *cons = (constr_t *)malloc(((size_t)S + 1) * sizeof(constr_t));
    for (long s = 0; s < S; s++) { cons[s].type = C_NONE; cons[s].refidx = 0; }
    int err = 0;
    int cur = 0, lastph = 0;   /* getStartPhase: Ref */

    if (p->doPrePhasing) {   /* Target.cpp:324-438 */
        beam_t B;
        beam_setup(&B, (int)hist_len(p->hsize_fast, p->hist), p->beamwidth_fast, p->delta_fast, p, cmd, (int)S,
                   calls, (int)ncalls, tg, cons, &pv, 0);
        if (S > 0) { cons[0].type = C_HETKEEP; cons[0].refidx = 0; }
        mmheap callheap, homheap; hp_init(&callheap); hp_init(&homheap);
        size_t nci = 1;
        for (long si = 1; si < S && !err; si++) {
            if ((int64_t)si == calls[nci]) {
                float pr = (float)((double)beam_call_keep(&B, (int)nci, 0) - 0.5);
                int ref = cur;
                constr_t c = {C_NONE, (int)(calls[nci] - calls[nci - 1] - 1)};
                if (nci > 1) {
                    float p2 = (float)((double)beam_call_keep(&B, (int)nci, 1) - 0.5);
                    if (fabsf(p2) > fabsf(pr)) { pr = p2; ref = lastph; c.refidx = (int)(calls[nci] - calls[nci - 2] - 1); }
                }
                lastph = cur;
                if (pr < 0.0f) { cur = !ref; c.type = C_HETSWITCH; }
                else { cur = ref; c.type = C_HETKEEP; }
                cons[si] = c;
                pr = fabsf(pr);
                hp_push(&callheap, pr, (int)si, 0);
                nci++;
            } else {
                float pr = beam_call_dosage(&B, (int)si);
                if (tg[si] == 0) { cons[si].type = C_HOMREF; cons[si].refidx = 0; pr = (float)(2.0 - (double)pr); }
                else { cons[si].type = C_HOMALT; cons[si].refidx = 0; }
                hp_push(&homheap, pr, (int)si, 0);
            }
            if (B.error) err = -1;
        }
        size_t smin = (size_t)((float)callheap.n * p->minfixsize);
        size_t smax = (size_t)((double)callheap.n * (1.0 - (double)p->maxfixsize));
        size_t si;
        for (si = 0; si < smin; si++) {
            hel cc = hp_popmin(&callheap);
            if ((double)cc.key >= (double)p->maxfixthr - 0.5 || ((double)cc.key >= (double)p->minfixthr - 0.5 && si >= smax)) break;
            cons[cc.a].type = C_NONE;
        }
        if (si == smin) {
            for (; si < (size_t)callheap.n; si++) {
                hel cc = hp_popmin(&callheap);
                if (cc.key > 0.0f) break;
                cons[cc.a].type = C_NONE;
            }
        }
        smin = (size_t)((float)homheap.n * p->minfixsize);
        smax = (size_t)((double)homheap.n * (1.0 - (double)p->maxfixsize));
        for (si = 0; si < smin; si++) {
            hel cc = hp_popmin(&homheap);
            if ((double)cc.key >= (double)p->maxfixthr * 2.0 || ((double)cc.key >= (double)p->minfixthr * 2.0 && si >= smax)) break;
            cons[cc.a].type = C_NONE;
        }
        hp_free(&callheap); hp_free(&homheap);
        beam_free(&B);
    }

    cur = 0;
    float *phaseProbs = (float *)malloc((ncalls + 1) * sizeof(float));
    size_t nprobs = 0;
    phaseProbs[nprobs++] = 0.0f;
    if (!err) {   /* Target.cpp:458-599 */
        beam_t B;
        beam_setup(&B, (int)hist_len(p->hsize, p->hist), p->beamwidth, p->delta, p, cmd, (int)S,
                   calls, (int)ncalls, tg, cons, &pv, 0);
        size_t m = 0;
        size_t stop = S > 0 ? (size_t)splits[calls[0]] : M;
        for (; m < stop; m++) {
            int a = 0, b = 0;
            switch (gt[m]) {
            case 2: a = b = 1; dos_mat[m] = 1.0f; dos_pat[m] = 1.0f; break;
            case 1: a = 0; b = 1; dos_mat[m] = 0.5f; dos_pat[m] = 0.5f; break;
            default: break;   /* HomRef; Miss without impMissing */
            }
            if (a) setbit(mat, m);
            if (b) setbit(pat, m);
        }
        if (m < M) {
            if (cur) setbit(mat, m); else setbit(pat, m);
            m++;
        }
        size_t nci = 1;
        for (; m < M && !err; m++) {
            int a = 0, b = 0;
            switch (gt[m]) {
            case 1:
                if (!getbit(monos, m)) {
                    float pr = (float)((double)beam_call_keep(&B, (int)nci, 0) - 0.5);
                    if (B.error) { err = -1; break; }
                    int ref = cur;
                    phaseProbs[nprobs++] = pr;
                    cur = pr < 0.0f ? !ref : ref;
                    nci++;
                } else {
                    dos_mat[m] = 0.5f; dos_pat[m] = 0.5f;
                }
                a = cur; b = !cur;
                break;
            case 2: a = b = 1; dos_mat[m] = 1.0f; dos_pat[m] = 1.0f; break;
            default: break;
            }
            if (a) setbit(mat, m);
            if (b) setbit(pat, m);
        }
        beam_free(&B);
    }

    float *callConfs = NULL;
    if (!err && S > 0) {   /* Target.cpp:601-619 */
        callConfs = (float *)calloc(ncalls, sizeof(float));
        if (p->doRevPhasing) callConfs[ncalls - 1] = (float)((double)fabsf(phaseProbs[nprobs - 1]) + 0.5);
        else for (size_t i = 0; i < nprobs && i < ncalls; i++) callConfs[i] = (float)((double)fabsf(phaseProbs[i]) + 0.5);
    }
    if (!err && p->doRevPhasing && S > 0) {   /* Target.cpp:620-758 */
        constr_t *rc = (constr_t *)malloc((size_t)S * sizeof(constr_t));
        for (long s = 0; s < S; s++) { rc[s].type = C_NONE; rc[s].refidx = 0; }
        for (long ci = 1; ci < S; ci++) {
            constr_t *c = &cons[ci];
            if (c->type == C_HETKEEP || c->type == C_HETSWITCH) {
                constr_t *r = &rc[ci - c->refidx - 1];
                if (r->type != C_NONE) {
                    long ridx = ci - c->refidx + r->refidx;
                    rc[ridx].refidx = c->refidx - r->refidx - 1;
                    rc[ridx].type = (c->type != r->type) ? C_HETSWITCH : C_HETKEEP;
                } else { r->type = c->type; r->refidx = c->refidx; }
            } else if (c->type == C_HOMREF || c->type == C_HOMALT) {
                rc[ci].type = c->type;
            }
        }
        rc[S - 1].type = C_HETKEEP; rc[S - 1].refidx = 0;
        float last = phaseProbs[nprobs - 1];
        float dref = last < 0.0f ? (float)(0.5 + (double)last) : (float)(0.5 - (double)last);
        float dalt = last < 0.0f ? (float)(0.5 - (double)last) : (float)(0.5 + (double)last);
        size_t site = (size_t)splits[calls[ncalls - 1]];
        dos_mat[site] = cur == 0 ? dref : dalt;
        dos_pat[site] = cur == 0 ? dalt : dref;
        pbwt_v rpv = pv;
        beam_t B;
        beam_setup(&B, (int)hist_len(p->hsize, p->hist), p->beamwidth, p->delta, p, cmd, (int)S,
                   calls, (int)ncalls, tg, rc, &rpv, 1);
        for (long rci = (long)ncalls - 2; rci >= 0 && !err; rci--) {
            float pr = (float)((double)beam_call_keep(&B, (int)rci, 0) - 0.5);
            if (B.error) { err = -1; break; }
            int ref = cur;
            if (fabsf(phaseProbs[rci + 1]) > fabsf(pr)) pr = phaseProbs[rci + 1];
            cur = pr < 0.0f ? !ref : ref;
            size_t s2 = (size_t)splits[calls[rci]];
            if (cur) { setbit(mat, s2); clrbit(pat, s2); } else { clrbit(mat, s2); setbit(pat, s2); }
            dref = pr < 0.0f ? (float)(0.5 + (double)pr) : (float)(0.5 - (double)pr);
            dalt = pr < 0.0f ? (float)(0.5 - (double)pr) : (float)(0.5 + (double)pr);
            dos_mat[s2] = cur == 0 ? dref : dalt;
            dos_pat[s2] = cur == 0 ? dalt : dref;
            callConfs[rci] = (float)((double)fabsf(pr) + 0.5);
        }
        beam_free(&B);
        free(rc);
    }
    if (!err && S > 0) {   /* Target.cpp:761-772 */
        float tc = 0.0f;
        for (size_t i = 0; i < ncalls; i++) tc = tc + callConfs[i];
        *totalconf = tc;
        *ncallsites = ncalls;
    }
    free(callConfs); free(phaseProbs); free(cons); free(tg); free(pb); free(cref); free(count0);
    free(cmd); free(calls); free(splits); free(monos); free(bh); free(gtw);
    return err;
}

int eo_phase_many(const uint8_t *gt, size_t n, const uint64_t *hapmajor, const uint64_t *sitemajor,
                  const float *cm, size_t M, size_t nhaps, const eo_phase_params *p, int nthreads,
                  uint64_t *mats, uint64_t *pats, float *dos_mats, float *dos_pats) {
    size_t wM = eo_W(M);
    int err = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads) reduction(| : err)
    for (long t = 0; t < (long)n; t++) {
        float tc; size_t nc;
        err |= eo_phase(gt + t * M, hapmajor, sitemajor, cm, M, nhaps, p, mats + t * wM, pats + t * wM,
                        dos_mats + t * M, dos_pats + t * M, &tc, &nc);
    }
    return err;
}
