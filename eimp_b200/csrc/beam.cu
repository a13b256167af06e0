// Eagle2-style beam phasing over the condensed PBWT, one warp per target.
//
// Device restatement of Target::phaseExtPBWT (Target.cpp:291-777) with Beam
// (Beam.cpp:41-837), BeamPath (BeamPath.cpp:29-291), HaplotypePath
// (HaplotypePath.cpp:36-483), BooleanHistory (BooleanHistory.cpp:31-113),
// History (History.h:29-81) and MinMaxHeap (MinMaxHeap.h:29-214).
//
// Work split inside the warp:
//  * haplotype-path extensions (the PBWT interval mappings over the history,
//    the bulk of the work) run one path per lane against the cursor's two
//    PBWT rows, which the warp stages in shared memory at every advance.  Each
//    path's probabilities are accumulated in its own lane in the reference's
//    order.  The reference copies intervals from the previously extended path
//    (HaplotypePath.cpp:330-390); they are recomputed here, which gives the
//    same intervals: an interval depends only on the recent history the two
//    paths share;
//  * beam-path extensions run one path per lane (per-path products; the
//    maximum and the reference counts do not depend on the order);
//  * the new list orders (haplotype paths after applying, beam paths after
//    applying and merging) are computed with warp scans; the positions are
//    the ones the reference's sequential loops produce;
//  * what depends on the sequential order stays on lane 0: the min-max heap
//    of the pruning, the merge of beam paths that share both histories (only
//    the duplicates, in list order), and the float sums of the calls and of
//    the recombination distances (over per-path terms the lanes prepare).
// Floating point follows the reference operation by operation: float
// arithmetic with explicit double where the reference promotes (pow(), double
// literals, std::ilogb), explicit round-to-nearest intrinsics (no FMA).
//
// The beam (two list buffers) and the per-warp scalars live in shared memory.
// The haplotype-path records, their probability rings and a pool of interval
// buffers (a path owns three: its intervals and its two extensions; copying a
// path hands over a buffer instead of copying it), and the constraint and
// probability vectors of the target live in an arena in global memory.
#include <climits>

#include "common.cuh"
#include "kernels.h"

namespace eimp {

namespace {

enum { C_HOMREF = 0, C_HETKEEP = 1, C_HETSWITCH = 2, C_HOMALT = 3, C_NONE = 4 };

struct Cons { int type, refidx; };

constexpr int PHMAX = 128;   // History<fp_type> ring (power of two >= H, H <= 128)
constexpr int PMAX = 128;    // largest beam width
constexpr int BPMAX = PMAX;  // beam paths held between two prunes (<= P)
constexpr int HTS_BITS = 8;
constexpr int HTS = 1 << HTS_BITS;   // merge hash table entries (load <= 1/2)
static_assert(BPMAX < HTS, "the merge table must never fill");

struct HPh {   // HaplotypePath
    unsigned long long d0, d1;   // BooleanHistory data (fill mask applied)
    int last;
    float p;
    int scaleexp;
    int niv, next0, next1;       // lengths of pbwtInt and of the two extension vectors
    float extp0, extp1;
    int extscaleexp;
    int refcnt0, refcnt1;
    int phstart;
    int biv, bext0, bext1;       // interval buffer ids
    unsigned char active0, active1, toext0, toext1;
};

struct BPh {   // BeamPath, 48 bytes
    unsigned short mat, pat;     // haplotype-path ids (< 4P + 8)
    float prob, weight;
    int nErr;
    float pErrPath, pErrPathp1;
    float extp[4];
    unsigned char active[4];
    signed char actidx;          // -2..3
    unsigned char extgeno;       // 0..3
};
static_assert(sizeof(BPh) == 48, "beam paths stay 48 bytes");

struct Hel { float key; int a; int b; };

struct __align__(16) WS {   // per-warp state in shared memory
    float prec[PHMAX];
    float cdv[PHMAX];
    Hel *heap;                    // the pruning's fallback heap: PMAX + 2 entries in the arena
    int2 ht[HTS];                 // merge keys: (key, surviving beam path), x = -1 when free
    BPh bp[2][BPMAX];             // the beam in list order (two buffers)
    float acc0[BPMAX], acc1[BPMAX];
    short slot[BPMAX];            // hash slot of each beam path during a merge
    unsigned char delmask[BPMAX]; // extensions the pruning deleted, per beam path
    int cursor, curridx, refidx, reverse;
    int nbp, bpsel, nhap, nfree, nivfree, err;
    int H, P, Delta, phsize;
    unsigned long long fill0, fill1;
    int histlast;
    int ires, ires2;
    int wse, delerr;   // weightScaleExp and deleteErr of the last prune (Beam.cpp:673-678)
    int c0inc, c0ref;  // zero counts of the cursor's two PBWT rows
    float fres;
    const Cons *constr;
    uint32_t *rowinc, *rowref;   // the cursor's PBWT rows (shared memory after the WS array)
    short *canon;                // per list position: first position of its run of equal histories
};

struct Ctx {
    // arena
    HPh *hp;
    float *ph;
    uint32_t *ivpool;            // intervals [l, r] packed l | r << 16 (K <= 65536)
    int *ivfree;
    int *happ, *happ_old;
    int2 *hapmap;
    int *fstack;
    int *copies;
    int NH, HMAX;
    // pbwt of this target
    const uint32_t *rows;
    const int32_t *count0;
    int Mp, K, kw;
    float Kinv;
    // condensed target
    const float *cmd;
    int S;
    const int32_t *calls;
    int ncalls;
    const uint8_t *tg;
    float pErr, pLimit, expectIBDcM;
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

// std::ilogb(float) as glibc defines it: the unbiased exponent (subnormals
// included), INT_MIN for zero and NaN, INT_MAX for infinity
__device__ __forceinline__ int ilogb_exact(float x) {
    const unsigned u = __float_as_uint(x) & 0x7fffffffu;
    if (u == 0) return INT_MIN;
    if (u >= 0x7f800000u) return u == 0x7f800000u ? INT_MAX : INT_MIN;
    const int e = (int)(u >> 23);
    if (e == 0) return (31 - __clz(u)) - 149;
    return e - 127;
}
// pow(2, n) for an integer n, exact
__device__ __forceinline__ double pow2i(int n) { return ldexp(1.0, n); }

// ------------------------------------------------------------------ histories
__device__ __forceinline__ void bh_push(HPh &h, int b, const WS &w) {   // BooleanHistory.cpp:55-70
    unsigned long long c0 = h.d0 >> 63;
    h.d0 = (h.d0 << 1) | (unsigned long long)(b ? 1 : 0);
    h.d1 = (h.d1 << 1) | c0;
    if (h.last != w.histlast) h.last++;
    h.d0 |= w.fill0;
    h.d1 |= w.fill1;
}
__device__ __forceinline__ int bh_at(const HPh &h, int pos) {
    return (int)(((pos < 64 ? h.d0 : h.d1) >> (pos & 63)) & 1ull);
}
__device__ __forceinline__ int bh_equal(const HPh &a, const HPh &b) {
    // BooleanHistory.cpp:91-97 compares a third 8-byte slot after the data
    // words, i.e. the members 'last' and 'histlast'
    return a.d0 == b.d0 && a.d1 == b.d1 && a.last == b.last;
}

__device__ __forceinline__ float *ph_ptr(const Ctx &c, int slot) { return c.ph + (size_t)slot * PHMAX; }
__device__ __forceinline__ uint32_t *iv_buf(const Ctx &c, int b) { return c.ivpool + (size_t)b * c.HMAX; }
// the interval lists hold non-empty intervals of positions < K <= 65536
__device__ __forceinline__ uint32_t iv_pack(int l, int r) { return (uint32_t)l | ((uint32_t)r << 16); }
__device__ __forceinline__ int iv_l(uint32_t v) { return (int)(v & 0xffffu); }
__device__ __forceinline__ int iv_r(uint32_t v) { return (int)(v >> 16); }

// ------------------------------------------------------------------ min-max heap (MinMaxHeap.h)
__device__ __forceinline__ int hlt(const Hel &x, const Hel &y) { return x.key < y.key; }
__device__ __forceinline__ void hswap(Hel *h, int i, int j) { Hel t = h[i]; h[i] = h[j]; h[j] = t; }
__device__ __forceinline__ int hminlevel(int i) { return ((31 - __clz(i + 1)) % 2) == 0; }
__device__ __forceinline__ int hpar(int i) { return (i - 1) / 2; }

__device__ void heap_bubble_helper(Hel *h, int i, int ismax) {
    while (i != 0) {
        int p = hpar(i);
        if (p == 0) return;
        int g = hpar(p);
        if (hlt(h[i], h[g]) ^ ismax) { hswap(h, g, i); i = g; }
        else return;
    }
}
__device__ void heap_push(Hel *h, int &n, float key, int a, int b) {
    h[n].key = key; h[n].a = a; h[n].b = b;
    int i = n++;
    if (i == 0) return;
    int p = hpar(i);
    if (hminlevel(i)) {
        if (hlt(h[p], h[i])) { hswap(h, p, i); heap_bubble_helper(h, p, 1); }
        else heap_bubble_helper(h, i, 0);
    } else {
        if (hlt(h[i], h[p])) { hswap(h, p, i); heap_bubble_helper(h, p, 0); }
        else heap_bubble_helper(h, i, 1);
    }
}
__device__ void heap_trickle(Hel *h, int n, int i) {
    const int ismax = hminlevel(i) ? 0 : 1;
    while (true) {
        int ext = i, lc = 2 * i + 1;
        if (lc < n && (hlt(h[lc], h[ext]) ^ ismax)) ext = lc;
        if (lc + 1 < n && (hlt(h[lc + 1], h[ext]) ^ ismax)) ext = lc + 1;
        int lg = 2 * lc + 1;
        for (int k = 0; k < 4 && lg + k < n; ++k)
            if (hlt(h[lg + k], h[ext]) ^ ismax) ext = lg + k;
        if (i == ext) return;
        hswap(h, i, ext);
        if (ext - lc > 1) {
            if (hlt(h[hpar(ext)], h[ext]) ^ ismax) hswap(h, hpar(ext), ext);
            i = ext;
        } else return;
    }
}
__device__ Hel heap_popmin(Hel *h, int &n) {
    Hel e = h[0];
    if (n == 1) { n = 0; return e; }
    hswap(h, 0, n - 1);
    n--;
    heap_trickle(h, n, 0);
    return e;
}
__device__ __forceinline__ int heap_maxidx(const Hel *h, int n) {
    if (n == 1) return 0;
    if (n == 2) return 1;
    return hlt(h[1], h[2]) ? 2 : 1;
}

// ------------------------------------------------------------------ haplotype paths
__device__ int ivbuf_alloc(const Ctx &c, WS &w) {
    if (w.nivfree == 0) { w.err |= EIMP_ERR_BEAM_CAPACITY; return 0; }
    return c.ivfree[--w.nivfree];
}

__device__ void hp_new(const Ctx &c, WS &w, int slot, int alt) {   // HaplotypePath.cpp:36-53 (lane 0)
    HPh &h = c.hp[slot];
    h.d0 = w.fill0; h.d1 = w.fill1; h.last = -1;
    bh_push(h, alt, w);
    h.p = 1.0f; h.scaleexp = 0;
    float *ph = ph_ptr(c, slot);
    for (int i = 0; i < w.phsize; i++) ph[i] = 0.0f;
    h.phstart = w.phsize - 1;
    ph[h.phstart] = 1.0f;
    h.niv = 0; h.next0 = 0; h.next1 = 0;
    h.extp0 = 0.0f; h.extp1 = 0.0f; h.extscaleexp = 0;
    h.refcnt0 = 0; h.refcnt1 = 0;
    h.active0 = h.active1 = h.toext0 = h.toext1 = 0;
    h.biv = ivbuf_alloc(c, w); h.bext0 = ivbuf_alloc(c, w); h.bext1 = ivbuf_alloc(c, w);
}

__device__ __forceinline__ void hp_mark_required(HPh &h, const Cons &cn) {   // HaplotypePath.cpp:139-158
    if (cn.type == C_NONE) { h.toext0 = 1; h.toext1 = 1; return; }
    int hb = bh_at(h, cn.refidx);
    if ((cn.type == C_HETKEEP && hb == 0) || (cn.type == C_HETSWITCH && hb == 1) || cn.type == C_HOMREF)
        h.toext0 = 1;
    else if ((cn.type == C_HETKEEP && hb == 1) || (cn.type == C_HETSWITCH && hb == 0) || cn.type == C_HOMALT)
        h.toext1 = 1;
}

// HaplotypePath::extend with updateScaling and calculateHaplotypeProbabilities
// (HaplotypePath.cpp:162-479) against the cursor's two PBWT rows in shared
// memory; returns extscaleexp.
//
// The history is walked in chunks of HXC steps: the chunk's intervals and
// probabilities are loaded together (the next chunk's loads are in flight
// while this one is computed) and the interval mappings of the chunk, pure
// functions of the loaded intervals, are computed before the sequential part
// that accumulates the probabilities, appends the extension intervals and
// stops at the first step where both extensions are empty, in the reference's
// order.  One step per chunk measured fastest on cfg2 (beam 67 ms against 74,
// 78, 83 and 93 ms for 2, 3, 4 and 6 steps): the smaller loop body costs the
// warps sharing an SM fewer instruction-fetch stalls than the deeper
// prefetch saves.
constexpr int HXC = 1;

__device__ int hp_extend(const Ctx &c, const WS &w, int slot) {
    HPh &h = c.hp[slot];
    float *ph = ph_ptr(c, slot);
    const int pm = w.phsize - 1;
    const int niv = h.niv, phstart = h.phstart;
    const int calc0 = h.toext0, calc1 = h.toext1;
    const uint32_t *iv = iv_buf(c, h.biv);
    uint32_t *e0 = iv_buf(c, h.bext0);
    uint32_t *e1 = iv_buf(c, h.bext1);
    int ns = h.scaleexp;
    {   // updateScaling (:224-258)
        const int e = ilogb_exact(h.p);
        if (abs(e) >= 20) {
            ns += e;
            const double f = pow2i(-e);
            for (int i = 0; i <= niv; i++) {
                float *x = &ph[(i + phstart) & pm];
                *x = (float)((double)*x * f);
            }
        }
        h.extscaleexp = ns;
    }
    const int lim = w.H < niv + 1 ? w.H : niv + 1;
    float p0 = 0.0f, p1 = 0.0f;
    int n0 = 0, n1 = 0;
    uint32_t last0 = 0u, last1 = 0u;   // the last entries appended (read only after an append)
    const int cnt0 = w.c0ref;
    const float t0 = __fmul_rn(ph[phstart & pm], w.prec[0]);
    if (cnt0 > 0) {
        if (calc0) p0 = __fmul_rn((float)cnt0, t0);
        last0 = iv_pack(0, cnt0 - 1);
        e0[n0++] = last0;
    }
    if (cnt0 < c.K) {
        if (calc1) p1 = __fmul_rn((float)(c.K - cnt0), t0);
        last1 = iv_pack(cnt0, c.K - 1);
        e1[n1++] = last1;
    }
    const uint32_t *rinc = w.rowinc, *rref = w.rowref;
    const int cinc = w.c0inc;
    uint32_t prevfrom = 0u;   // compared only from the second step on
    uint32_t fr[HXC], nfr[HXC];
    float tph[HXC], ntph[HXC];
#pragma unroll
    for (int j = 0; j < HXC; j++)
        if (1 + j < lim) { fr[j] = iv[j]; tph[j] = ph[(1 + j + phstart) & pm]; }
    bool stop = false;
    for (int base = 1; base < lim && !stop; base += HXC) {
        const int nb = base + HXC;
#pragma unroll
        for (int j = 0; j < HXC; j++)   // the next chunk's loads
            if (nb + j < lim) { nfr[j] = iv[nb + j - 1]; ntph[j] = ph[(nb + j + phstart) & pm]; }
        // mappings of the chunk's intervals; a step whose interval equals the
        // previous step's takes the reference's reuse branch below and needs
        // none (about 60 % of the steps, mostly the same for all lanes)
        int A0[HXC], B0[HXC], A1[HXC], B1[HXC];
#pragma unroll
        for (int j = 0; j < HXC; j++) {
            A0[j] = 0; B0[j] = -1; A1[j] = 0; B1[j] = -1;
            const uint32_t pf = j == 0 ? prevfrom : fr[j - 1];
            const bool same = base + j > 1 && pf == fr[j];
            if (base + j < lim && !same) {
                int cl, cr, il, ir;
                pbwt_map(rinc, cinc, iv_l(fr[j]), iv_r(fr[j]), cl, cr, il, ir);
                pbwt_map(rref, cnt0, cl, cr, A0[j], B0[j], A1[j], B1[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < HXC; j++) {
            const int i = base + j;
            if (stop || i >= lim) break;
            const uint32_t from = fr[j];
            int a0 = A0[j], b0 = B0[j], a1 = A1[j], b1 = B1[j];
            if (i > 1 && prevfrom == from) {   // :395-399
                a0 = 0; b0 = -1; a1 = 0; b1 = -1;
                if (n0 == i) { a0 = iv_l(last0); b0 = iv_r(last0); }
                if (n1 == i) { a1 = iv_l(last1); b1 = iv_r(last1); }
            }
            prevfrom = from;
            const float ti = __fmul_rn(tph[j], w.prec[i]);
            bool any = false;
            if (a0 <= b0) {
                if (calc0) p0 = __fadd_rn(p0, __fmul_rn((float)(b0 - a0 + 1), ti));
                last0 = iv_pack(a0, b0);
                e0[n0++] = last0;
                any = true;
            }
            if (a1 <= b1) {
                if (calc1) p1 = __fadd_rn(p1, __fmul_rn((float)(b1 - a1 + 1), ti));
                last1 = iv_pack(a1, b1);
                e1[n1++] = last1;
                any = true;
            }
            if (!any) stop = true;
        }
#pragma unroll
        for (int j = 0; j < HXC; j++) { fr[j] = nfr[j]; tph[j] = ntph[j]; }
    }
    h.next0 = n0; h.next1 = n1;
    h.extp0 = p0; h.extp1 = p1;
    h.active0 = calc0; h.active1 = calc1;
    return ns;
}

// HaplotypePath::applyExtension (HaplotypePath.cpp:77-103)
__device__ void hp_apply(const Ctx &c, const WS &w, int slot, int e) {
    HPh &h = c.hp[slot];
    bh_push(h, e, w);
    h.p = e ? h.extp1 : h.extp0;
    h.scaleexp = h.extscaleexp;
    float *ph = ph_ptr(c, slot);
    h.phstart = (h.phstart - 1) & (w.phsize - 1);
    ph[h.phstart] = h.p;
    int t = h.biv;
    if (e) { h.biv = h.bext1; h.bext1 = t; h.niv = h.next1; }
    else { h.biv = h.bext0; h.bext0 = t; h.niv = h.next0; }
    h.next0 = 0; h.next1 = 0;
    h.extp0 = 0.0f; h.extp1 = 0.0f; h.extscaleexp = 0;
    h.active0 = h.active1 = h.toext0 = h.toext1 = 0;
    h.refcnt0 = 0; h.refcnt1 = 0;
}

// ------------------------------------------------------------------ beam paths
__device__ __forceinline__ int incon_(int ext, int g) {   // BeamPath.cpp:246-274
    switch (g) {
    case 1: return ext == 0 || ext == 3;
    case 0: return ext > 0;
    case 2: return ext < 3;
    default: return 1;
    }
}
__device__ __forceinline__ void bp_update_errors(BPh &b, int ext, int delerr, float pErr) {   // BeamPath.cpp:209-228
    int add = (incon_(ext, b.extgeno) ? 1 : 0) - (delerr ? 1 : 0);
    b.nErr += add;
    if (add < 0) { b.pErrPathp1 = b.pErrPath; b.pErrPath = __fdiv_rn(b.pErrPath, pErr); }
    else for (int a = 0; a < add; a++) { b.pErrPath = b.pErrPathp1; b.pErrPathp1 = __fmul_rn(b.pErrPathp1, pErr); }
}
__device__ __forceinline__ void bp_update_actidx(BPh &b) {
    b.actidx = -1;
    for (int i = 3; i >= 0; i--) if (b.active[i]) { b.actidx = i; break; }
}
__device__ __forceinline__ int bp_next_active(const BPh &b, int x) {
    for (int i = x - 1; i >= 0; i--) if (b.active[i]) return i;
    return -1;
}
__device__ __forceinline__ void bp_single(BPh &b, int id, float p1, float p2, float scale, int incon, float &maxP) {
    float x = __fmul_rn(__fmul_rn(p1, p2), scale);
    x = __fmul_rn(x, incon ? b.pErrPathp1 : b.pErrPath);
    b.extp[id] = x;
    if (maxP < x) maxP = x;
    b.active[id] = 1;
    b.actidx = id;
}

// BeamPath::extend (BeamPath.cpp:121-197); reference counts by atomics
__device__ float bp_extend(const Ctx &c, BPh &b, int g, const Cons &cn, int bpscaleexp) {
    b.extgeno = g;
    HPh &pm = c.hp[c.happ[b.mat]];
    HPh &pp = c.hp[c.happ[b.pat]];
    const float pm0 = pm.extp0, pm1 = pm.extp1, pp0 = pp.extp0, pp1 = pp.extp1;
    const int c0 = pm.active0, c1 = pm.active1, d0 = pp.active0, d1 = pp.active1;
    const float scale = (float)pow2i(pm.extscaleexp + pp.extscaleexp + bpscaleexp);
    float maxP = 0.0f;
    const int t = cn.type;
    const int hb = (t == C_HETKEEP || t == C_HETSWITCH) ? bh_at(pm, cn.refidx) : 0;
    if (t == C_NONE || t == C_HOMREF) {
        if (c0 && d0) { bp_single(b, 0, pm0, pp0, scale, incon_(0, g), maxP); atomicAdd(&pm.refcnt0, 1); atomicAdd(&pp.refcnt0, 1); }
    }
    if (t == C_NONE || (t == C_HETKEEP && hb == 0) || (t == C_HETSWITCH && hb == 1)) {
        if (c0 && d1) { bp_single(b, 1, pm0, pp1, scale, incon_(1, g), maxP); atomicAdd(&pm.refcnt0, 1); atomicAdd(&pp.refcnt1, 1); }
    }
    if (t == C_NONE || (t == C_HETKEEP && hb == 1) || (t == C_HETSWITCH && hb == 0)) {
        if (c1 && d0) { bp_single(b, 2, pm1, pp0, scale, incon_(2, g), maxP); atomicAdd(&pm.refcnt1, 1); atomicAdd(&pp.refcnt0, 1); }
    }
    if (t == C_NONE || t == C_HOMALT) {
        if (c1 && d1) { bp_single(b, 3, pm1, pp1, scale, incon_(3, g), maxP); atomicAdd(&pm.refcnt1, 1); atomicAdd(&pp.refcnt1, 1); }
    }
    return maxP;
}


// BeamPath::markExtensionDeleted (BeamPath.cpp:101-112) on the beam path; the
// haplotype-path side is applied after the heap pass from delmask
__device__ __forceinline__ void bp_mark_deleted_deferred(WS &w, BPh &b, int it, int ext) {
    b.active[ext] = 0;
    bp_update_actidx(b);
    w.delmask[it] |= (unsigned char)(1u << ext);
}

// ------------------------------------------------------------------ beam
// Beam::calculateRecProbs (Beam.cpp:541-573).  The distance to history entry
// i is the float sum of the i preceding split-site distances (lane 0, in the
// reference's order); the probabilities are per entry (lanes).
__device__ void beam_calc_rec(const Ctx &c, WS &w) {
    const int lane = lane_id();
    const int cur = w.cursor;
    const int L = w.reverse ? min(w.H, c.S - cur) : min(w.H, cur + 1);
    for (int i = lane; i < L; i += 32) w.cdv[i] = c.cmd[w.reverse ? cur + 1 + i : cur - i];
    __syncwarp();
    if (lane == 0) {
        float cd = 0.0f;
        int i = 0;
        for (; i + 4 <= L; i += 4) {
            const float4 x = *reinterpret_cast<const float4 *>(&w.cdv[i]);
            w.cdv[i] = cd; cd = __fadd_rn(cd, x.x);
            w.cdv[i + 1] = cd; cd = __fadd_rn(cd, x.y);
            w.cdv[i + 2] = cd; cd = __fadd_rn(cd, x.z);
            w.cdv[i + 3] = cd; cd = __fadd_rn(cd, x.w);
        }
        for (; i < L; i++) { const float x = w.cdv[i]; w.cdv[i] = cd; cd = __fadd_rn(cd, x); }
    }
    __syncwarp();
    const float cursordiff = w.reverse ? c.cmd[cur] : c.cmd[cur + 1];
    for (int i = lane; i < L; i += 32) {
        const float cd = w.cdv[i];
        float tmp1 = (float)(1.0 + (double)__fdiv_rn(cd, c.expectIBDcM));
        float pr = (float)(1.0 / (double)__fmul_rn(tmp1, tmp1));
        float tmp2 = (float)(1.0 + (double)__fdiv_rn(__fadd_rn(cd, cursordiff), c.expectIBDcM));
        pr = (float)((double)pr - 1.0 / (double)__fmul_rn(tmp2, tmp2));
        pr = fmaxf(fminf(pr, 1.0f), 0.000001f);
        w.prec[i] = __fmul_rn(pr, c.Kinv);
    }
    __syncwarp();
}

// the cursor's two PBWT rows (the incon row of the previous split site and
// the ref row of this one) into shared memory
__device__ void beam_load_rows(const Ctx &c, WS &w) {
    const int cur = w.cursor;
    const int mi = w.reverse ? 2 * (cur + 1) : 2 * cur, mr = 2 * cur + 1;
    const int pi = w.reverse ? 2 * c.Mp - 1 - mi : mi, pr = w.reverse ? 2 * c.Mp - 1 - mr : mr;
    const uint2 *si = reinterpret_cast<const uint2 *>(c.rows + (size_t)pi * c.kw);
    const uint2 *sr = reinterpret_cast<const uint2 *>(c.rows + (size_t)pr * c.kw);
    uint2 *di = reinterpret_cast<uint2 *>(w.rowinc), *dr = reinterpret_cast<uint2 *>(w.rowref);
    const int n2 = c.kw / 2;
    for (int i = lane_id(); i < n2; i += 32) { di[i] = si[i]; dr[i] = sr[i]; }
    if (lane_id() == 0) { w.c0inc = c.count0[mi]; w.c0ref = c.count0[mr]; }
    __syncwarp();
}

__device__ void beam_init(const Ctx &c, WS &w, const Cons *constr, int reverse, int H, int P, int Delta) {
    const int lane = lane_id();
    for (int i = lane; i < c.NH; i += 32) c.fstack[i] = c.NH - 1 - i;
    for (int i = lane; i < 3 * c.NH; i += 32) c.ivfree[i] = 3 * c.NH - 1 - i;
    for (int i = lane; i < HTS; i += 32) w.ht[i] = make_int2(-1, INT_MAX);
    for (int i = lane; i < PHMAX; i += 32) w.prec[i] = 0.0f;
    __syncwarp();
    if (lane == 0) {   // Beam.cpp:41-92
        w.H = H; w.P = P; w.Delta = Delta;
        int l2 = 31 - __clz(H);
        if ((1 << l2) != H) l2++;
        w.phsize = 1 << l2;
        w.histlast = H - 1;
        int lw = (H - 1) / 64;
        unsigned long long mlw = (H % 64 == 0) ? 0ull : ~((1ull << (H % 64)) - 1ull);
        w.fill0 = 0 < lw ? 0ull : (0 == lw ? mlw : ~0ull);
        w.fill1 = 1 < lw ? 0ull : (1 == lw ? mlw : ~0ull);
        w.reverse = reverse;
        w.constr = constr;
        w.cursor = reverse ? c.S : -1;
        w.curridx = -1; w.refidx = -1;
        w.err = 0;
        w.nfree = c.NH;
        w.nivfree = 3 * c.NH;
        int mat = c.fstack[--w.nfree], pat = c.fstack[--w.nfree];
        hp_new(c, w, mat, 0);
        hp_new(c, w, pat, 1);
        c.happ[0] = mat; c.happ[1] = pat;
        w.nhap = 2;
        w.bpsel = 0;
        BPh &b = w.bp[0][0];
        b.mat = 0; b.pat = 1; b.weight = 1.0f;
        b.nErr = 0; b.pErrPath = 1.0f; b.pErrPathp1 = __fmul_rn(1.0f, c.pErr);
        b.prob = (float)(pow2i(0) * (double)c.hp[mat].p * (double)c.hp[pat].p * 1.0);
        for (int i = 0; i < 4; i++) { b.extp[i] = 0.0f; b.active[i] = 0; }
        b.actidx = -1; b.extgeno = 3;
        w.nbp = 1;
    }
    __syncwarp();
}

__device__ __forceinline__ float warp_minf(float v) {
    for (int o = 16; o; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_maxf(float v) {
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_mini(int v) {
    for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_maxi(int v) {
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_sumi(int v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Beam::prunePaths (Beam.cpp:577-787), the filter and the min-max heap.  The
// candidates are, per beam path in list order, the extension indices from
// the active index down to 0 (unconstrained) or the active index alone.
//
// The reference streams the candidates at or above the limit through a
// min-max heap of capacity P that replaces its minimum only by a strictly
// larger key.  When at most P candidates reach the limit nothing is evicted;
// when more do but the P-th largest key is strictly larger than the
// (P+1)-th, the heap ends holding exactly the P largest (every candidate
// outside it is at most the final minimum, every one inside at least).  In
// both cases the lanes decide everything: the P-th largest key comes from a
// bitwise search over the keys (non-negative floats order like their bit
// patterns), and the heap's minimum and maximum are a survivor with the
// smallest and one with the largest key, provided all survivors tied at the
// smallest key give the same weightScaleExp and all tied at the largest the
// same deleteErr (else which tied element the heap holds at its root would
// matter).  Otherwise lane 0 runs the heap in the reference's order.  The
// reference counts of the haplotype paths are decremented afterwards by the
// lanes (nothing in the selection reads them).  Returns 0 when no extension
// survives.
constexpr int PRR = (BPMAX + 31) / 32;   // beam paths per lane

__device__ __forceinline__ unsigned key_bits(float p) { return p == 0.0f ? 0u : __float_as_uint(p); }

__device__ int beam_prune_select(const Ctx &c, WS &w, float maxP, const Cons &cn) {
    const int lane = lane_id();
    BPh *bp = w.bp[w.bpsel];
    const int nbp = w.nbp, P = w.P;
    const float limit = __fmul_rn(c.pLimit, maxP);
    const bool allext = cn.type == C_NONE;
    for (int it = lane; it < nbp; it += 32) w.delmask[it] = 0;
    // the candidates at or above the limit: bit 4r+ex of sel for extension ex
    // of beam path lane+32r (their keys are read back from shared memory)
    unsigned sel = 0;
    float kmin = __int_as_float(0x7f800000), kmax = -__int_as_float(0x7f800000);
#pragma unroll
    for (int r = 0; r < PRR; r++) {
        const int it = lane + 32 * r;
        const BPh *b = &bp[it < nbp ? it : 0];
        const int ai = it < nbp ? b->actidx : -1;
#pragma unroll
        for (int ex = 0; ex < 4; ex++) {
            if (ex <= ai && (allext || ex == ai)) {
                const float p = b->extp[ex];
                if (p >= limit) {
                    sel |= 1u << (4 * r + ex);
                    kmin = fminf(kmin, p); kmax = fmaxf(kmax, p);
                }
            }
        }
    }
    const int nA = warp_sumi(__popc(sel));
    kmin = warp_minf(kmin);
    kmax = warp_maxf(kmax);
    // survivors: the selected candidates with key >= thr
    unsigned thr = 0u;
    bool fast = true;
    if (nA > P) {
        for (int bit = 31; bit >= 0; bit--) {
            const unsigned cand = thr | (1u << bit);
            int cnt = 0;
#pragma unroll 1
            for (int q = 0; q < PRR * 4; q++) cnt += ((sel >> q) & 1u) && key_bits(bp[lane + 32 * (q >> 2)].extp[q & 3]) >= cand;
            if (warp_sumi(cnt) >= P) thr = cand;
        }
        int cnt = 0;
#pragma unroll 1
        for (int q = 0; q < PRR * 4; q++) cnt += ((sel >> q) & 1u) && key_bits(bp[lane + 32 * (q >> 2)].extp[q & 3]) >= thr;
        fast = warp_sumi(cnt) == P;   // else ties straddle the P-th place
    }
    unsigned surv = sel;
    if (thr)
#pragma unroll 1
        for (int q = 0; q < PRR * 4; q++)
            if (((sel >> q) & 1u) && key_bits(bp[lane + 32 * (q >> 2)].extp[q & 3]) < thr) surv &= ~(1u << q);
    int wse = 0, delerr = 0;
    const int nsurv = nA > P ? P : nA;
    if (fast && nsurv > 0) {
        const unsigned kminb = nA > P ? thr : key_bits(kmin), kmaxb = key_bits(kmax);
        int lo0 = INT_MAX, hi0 = INT_MIN, lo1 = 1, hi1 = 0;
#pragma unroll 1
        for (int q = 0; q < PRR * 4; q++) {
            if (!((surv >> q) & 1u)) continue;
            const BPh &b = bp[lane + 32 * (q >> 2)];
            const unsigned kq = key_bits(b.extp[q & 3]);
            if (kq == kminb) { const int e = -ilogb_exact(b.weight); lo0 = min(lo0, e); hi0 = max(hi0, e); }
            if (kq == kmaxb) { const int f = b.nErr > 0; lo1 = min(lo1, f); hi1 = max(hi1, f); }
        }
        lo0 = warp_mini(lo0); hi0 = warp_maxi(hi0);
        lo1 = warp_mini(lo1); hi1 = warp_maxi(hi1);
        fast = lo0 == hi0 && lo1 == hi1;
        wse = lo0;
        delerr = lo1;
    }
    __syncwarp();
    if (fast) {
#pragma unroll
        for (int r = 0; r < PRR; r++) {
            const int it = lane + 32 * r;
            if (it >= nbp) continue;
            BPh &b = bp[it];
            unsigned dm = 0;
            for (int ex = b.actidx; ex >= 0; ex = allext ? ex - 1 : -1)
                if (!((surv >> (4 * r + ex)) & 1u)) { b.active[ex] = 0; dm |= 1u << ex; }
            if (dm) { bp_update_actidx(b); w.delmask[it] = (unsigned char)dm; }
        }
        if (lane == 0) { w.ires = nsurv; w.wse = wse; w.delerr = delerr; }
    } else if (lane == 0) {
        Hel *hq = w.heap;
        int n = 0;
        for (int it = 0; it < nbp; it++) {
            BPh &b = bp[it];
            int ex = b.actidx;
            while (ex >= 0) {
                const float p = b.extp[ex];
                if (p >= limit) {
                    if (n < P || (n == P && p > hq[0].key)) {
                        if (n == P) {
                            Hel e = heap_popmin(hq, n);
                            bp_mark_deleted_deferred(w, bp[e.a], e.a, e.b);
                        }
                        heap_push(hq, n, p, it, ex);
                    } else bp_mark_deleted_deferred(w, b, it, ex);
                } else bp_mark_deleted_deferred(w, b, it, ex);
                ex = allext ? ex - 1 : -1;
            }
        }
        w.ires = n;
        if (n) {
            w.wse = -ilogb_exact(bp[hq[0].a].weight);                    // weightScaleExp
            w.delerr = bp[hq[heap_maxidx(hq, n)].a].nErr > 0;            // deleteErr
        }
    }
    __syncwarp();
    const int n = w.ires;
    // the deletions (HaplotypePath::markExtensionDeleted, HaplotypePath.cpp:
    // 105-109), aggregated per haplotype-path extension: a count reaches
    // zero (the extension becomes inactive) in exactly the decrement that
    // takes it from >= 1 to <= 0, however the decrements are grouped
    for (int it = lane; it < nbp; it += 32) {
        const unsigned dm = w.delmask[it];
        if (!dm) continue;
        HPh &pm = c.hp[c.happ[bp[it].mat]];
        HPh &pp = c.hp[c.happ[bp[it].pat]];
        const int dm0 = (int)(dm & 1u) + (int)((dm >> 1) & 1u);          // mat extension 0: ext 0, 1
        const int dm1 = (int)((dm >> 2) & 1u) + (int)((dm >> 3) & 1u);   // mat extension 1: ext 2, 3
        const int dp0 = (int)(dm & 1u) + (int)((dm >> 2) & 1u);          // pat extension 0: ext 0, 2
        const int dp1 = (int)((dm >> 1) & 1u) + (int)((dm >> 3) & 1u);   // pat extension 1: ext 1, 3
        const int om0 = dm0 ? atomicSub(&pm.refcnt0, dm0) : 0;
        const int om1 = dm1 ? atomicSub(&pm.refcnt1, dm1) : 0;
        const int op0 = dp0 ? atomicSub(&pp.refcnt0, dp0) : 0;
        const int op1 = dp1 ? atomicSub(&pp.refcnt1, dp1) : 0;
        if (dm0 && om0 >= 1 && om0 - dm0 <= 0) pm.active0 = 0;
        if (dm1 && om1 >= 1 && om1 - dm1 <= 0) pm.active1 = 0;
        if (dp0 && op0 >= 1 && op0 - dp0 <= 0) pp.active0 = 0;
        if (dp1 && op1 >= 1 && op1 - dp1 <= 0) pp.active1 = 0;
    }
    __syncwarp();
    return n > 0;
}

// apply the haplotype-path extensions (Beam.cpp:684-726).  The new list holds
// the paths extended with 0 in old order, then the paths extended with 1 in
// old order; a path with both extensions stays among the first and its copy
// (HaplotypePath.cpp:55-75), which takes the 1-extension, among the second.
// Positions come from warp scans; released slots are pushed before the copies
// take theirs (slot numbers are storage only and do not change results).
__device__ void beam_apply_hap(const Ctx &c, WS &w) {
    const int lane = lane_id();
    const unsigned FULL = 0xffffffffu;
    const int nold = w.nhap;
    for (int i = lane; i < nold; i += 32) c.happ_old[i] = c.happ[i];
    __syncwarp();
    int next0 = 0, nrel = 0, ncp = 0;
    for (int base = 0; base < nold; base += 32) {
        const int i = base + lane;
        bool a0 = false, a1 = false;
        if (i < nold) { const HPh &h = c.hp[c.happ_old[i]]; a0 = h.active0; a1 = h.active1; }
        next0 += __popc(__ballot_sync(FULL, a0));
        nrel += __popc(__ballot_sync(FULL, i < nold && !a0 && !a1));
        ncp += __popc(__ballot_sync(FULL, a0 && a1));
    }
    const int nfree0 = w.nfree, nivfree0 = w.nivfree;
    if (nfree0 + nrel < ncp || nivfree0 + 3 * nrel < 3 * ncp) {
        if (lane == 0) w.err |= EIMP_ERR_BEAM_CAPACITY;
        __syncwarp();
        return;
    }
    int zero = 0, one = next0, rel = 0, cp = 0;
    for (int base = 0; base < nold; base += 32) {
        const int i = base + lane;
        bool a0 = false, a1 = false;
        int id = -1;
        if (i < nold) { id = c.happ_old[i]; const HPh &h = c.hp[id]; a0 = h.active0; a1 = h.active1; }
        const unsigned b0 = __ballot_sync(FULL, a0), b1 = __ballot_sync(FULL, a1);
        const unsigned br = __ballot_sync(FULL, i < nold && !a0 && !a1), bc = __ballot_sync(FULL, a0 && a1);
        const unsigned lt = lanemask_lt();
        if (i < nold) {
            const int z = zero + __popc(b0 & lt), o = one + __popc(b1 & lt);
            c.hapmap[i] = make_int2(z, o);
            if (a0) c.happ[z] = id;
            else if (a1) c.happ[o] = id;
            if (!a0 && !a1) {
                const int r = rel + __popc(br & lt);
                const HPh &h = c.hp[id];
                c.fstack[nfree0 + r] = id;
                c.ivfree[nivfree0 + 3 * r] = h.biv;
                c.ivfree[nivfree0 + 3 * r + 1] = h.bext0;
                c.ivfree[nivfree0 + 3 * r + 2] = h.bext1;
            } else if (a0 && a1) {
                const int k = cp + __popc(bc & lt);
                c.copies[3 * k] = id;
                c.copies[3 * k + 2] = o;
            }
        }
        zero += __popc(b0); one += __popc(b1); rel += __popc(br); cp += __popc(bc);
    }
    __syncwarp();
    const int nf = nfree0 + nrel, nvf = nivfree0 + 3 * nrel;
    // records of the copies: the copy takes the extension-1 intervals as its
    // own; the source gets a fresh buffer for them
    for (int k = lane; k < ncp; k += 32) {
        const int id = c.copies[3 * k];
        const int slot = c.fstack[nf - 1 - k];
        c.copies[3 * k + 1] = slot;
        c.happ[c.copies[3 * k + 2]] = slot;
        HPh &o = c.hp[id];
        HPh &n = c.hp[slot];
        n.d0 = o.d0; n.d1 = o.d1; n.last = o.last;
        n.p = o.extp1; n.scaleexp = o.extscaleexp;
        n.phstart = o.phstart;
        n.biv = o.bext1; n.niv = o.next1;
        n.bext0 = c.ivfree[nvf - 1 - 3 * k];
        n.bext1 = c.ivfree[nvf - 2 - 3 * k];
        n.next0 = 0; n.next1 = 0;
        n.active0 = n.active1 = n.toext0 = n.toext1 = 0;
        n.refcnt0 = 0; n.refcnt1 = 0;
        n.extp0 = 0.0f; n.extp1 = 0.0f; n.extscaleexp = 0;
        o.bext1 = c.ivfree[nvf - 3 - 3 * k];
        o.next1 = 0;   // (the reference keeps a stale copy; it is rewritten before use)
    }
    if (lane == 0) { w.nfree = nf - ncp; w.nivfree = nvf - 3 * ncp; w.nhap = one; }
    __syncwarp();
    // probability rings of the copies: 16-byte pieces, one per lane, four
    // copies' loads in flight before their stores
    const int phs = w.phsize;
    if (phs >= 4) {
        const int n4 = phs / 4;
        for (int k0 = 0; k0 < ncp; k0 += 4) {
            float4 v[4];
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (k0 + j < ncp && lane < n4)
                    v[j] = reinterpret_cast<const float4 *>(ph_ptr(c, c.copies[3 * (k0 + j)]))[lane];
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (k0 + j < ncp && lane < n4)
                    reinterpret_cast<float4 *>(ph_ptr(c, c.copies[3 * (k0 + j) + 1]))[lane] = v[j];
        }
    } else {
        for (int k = 0; k < ncp; k++)
            if (lane < phs) ph_ptr(c, c.copies[3 * k + 1])[lane] = ph_ptr(c, c.copies[3 * k])[lane];
    }
    __syncwarp();
    // the copies: push bit 1 and the extension-1 probability
    for (int k = lane; k < ncp; k += 32) {
        const int slot = c.copies[3 * k + 1];
        HPh &n = c.hp[slot];
        bh_push(n, 1, w);
        float *ph = ph_ptr(c, slot);
        n.phstart = (n.phstart - 1) & (phs - 1);
        ph[n.phstart] = n.p;
    }
    // old paths still alive: apply their (single or zero) extension
    for (int i = lane; i < nold; i += 32) {
        const int id = c.happ_old[i];
        HPh &h = c.hp[id];
        if (!(h.active0 || h.active1)) continue;
        hp_apply(c, w, id, h.active0 ? 0 : 1);
    }
    __syncwarp();
}

__device__ __forceinline__ void bp_make(BPh &o, const BPh &b, int ex, int mat, int pat, int wse, double wsf,
                                        int delerr, float pErr) {   // BeamPath.cpp:44-96
    o.mat = mat; o.pat = pat;
    o.prob = b.extp[ex]; o.weight = b.weight;
    o.nErr = b.nErr; o.pErrPath = b.pErrPath; o.pErrPathp1 = b.pErrPathp1;
    o.extgeno = b.extgeno;
    if (wse != 0) o.weight = (float)((double)o.weight * wsf);
    bp_update_errors(o, ex, delerr, pErr);
    for (int q = 0; q < 4; q++) { o.extp[q] = 0.0f; o.active[q] = 0; }
    o.actidx = -1; o.extgeno = 3;
}

// apply the beam-path extensions (Beam.cpp:728-779): each path with a
// surviving extension keeps its position with its lowest extension; its other
// extensions are appended in the reference's order (paths in list order,
// extensions in descending index).  Positions come from warp scans.
__device__ void beam_apply_bp(const Ctx &c, WS &w) {
    const int lane = lane_id();
    const unsigned FULL = 0xffffffffu;
    const int wse = w.wse, delerr = w.delerr;
    const double wsf = pow2i(wse);
    const BPh *src = w.bp[w.bpsel];
    BPh *dst = w.bp[w.bpsel ^ 1];
    const int nbp = w.nbp;
    int nsurv = 0;
    for (int base = 0; base < nbp; base += 32) {
        const int it = base + lane;
        nsurv += __popc(__ballot_sync(FULL, it < nbp && src[it].actidx >= 0));
    }
    int k = 0, app = nsurv;
    for (int base = 0; base < nbp; base += 32) {
        const int it = base + lane;
        int nact = 0;
        if (it < nbp) {
            const BPh &b = src[it];
            nact = (int)b.active[0] + (int)b.active[1] + (int)b.active[2] + (int)b.active[3];
        }
        const unsigned bs = __ballot_sync(FULL, nact > 0);
        const int extra = nact > 0 ? nact - 1 : 0;
        int x = extra;   // inclusive scan of the extra extensions
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        const int tot = __shfl_sync(FULL, x, 31);
        if (nact > 0) {
            const BPh &b = src[it];
            const int2 mm = c.hapmap[b.mat], pm = c.hapmap[b.pat];
            const int mat[2] = {mm.x, mm.y}, pat[2] = {pm.x, pm.y};
            int pos = app + x - extra;
            int ex = b.actidx;
            for (int r = 0; r < extra; r++) {
                if (pos < BPMAX) bp_make(dst[pos], b, ex, mat[ex >> 1], pat[ex & 1], wse, wsf, delerr, c.pErr);
                pos++;
                ex = bp_next_active(b, ex);
            }
            bp_make(dst[k + __popc(bs & lanemask_lt())], b, ex, mat[ex >> 1], pat[ex & 1], wse, wsf, delerr,
                    c.pErr);
        }
        k += __popc(bs);
        app += tot;
    }
    if (lane == 0) {
        if (app > BPMAX) w.err |= EIMP_ERR_BEAM_CAPACITY;
        w.nbp = min(app, BPMAX);
        w.bpsel ^= 1;
    }
    __syncwarp();
}

// Beam::mergePaths (Beam.cpp:790-837).  Each beam path's key is the pair of
// first list positions of its two histories (runs of equal histories are
// adjacent in the list).  The first path of each key survives unless a later
// one with the same key is more probable; the duplicates are merged on lane
// 0 in list order (the reference's sequential order within each key), then
// the survivors are compacted into the other buffer.
__device__ void beam_merge(const Ctx &c, WS &w) {
    const int lane = lane_id();
    const unsigned FULL = 0xffffffffu;
    const int nhap = w.nhap;
    int carry = 0;
    for (int base = 0; base < nhap; base += 32) {
        const int i = base + lane;
        bool head = true;
        if (i < nhap && i > 0) head = !bh_equal(c.hp[c.happ[i]], c.hp[c.happ[i - 1]]);
        const unsigned hb = __ballot_sync(FULL, i < nhap && head);
        const unsigned upto = hb & (lane == 31 ? FULL : ((2u << lane) - 1u));
        const int cn = upto ? base + 31 - __clz(upto) : carry;
        if (i < nhap) w.canon[i] = (short)cn;
        carry = __shfl_sync(FULL, cn, 31);
    }
    __syncwarp();
    BPh *bp = w.bp[w.bpsel];
    const int n = w.nbp;
    bool anydup = false;
    for (int it = lane; it < n; it += 32) {
        const int mr = w.canon[bp[it].mat], pr = w.canon[bp[it].pat];
        const int k0 = mr < pr ? mr : pr, k1 = mr < pr ? pr : mr;
        const int key = (k0 << 16) | k1;
        int slot = (int)(((unsigned)key * 2654435761u) >> (32 - HTS_BITS)) & (HTS - 1);
        // linear probing; the table holds at most BPMAX < HTS keys, so a
        // free or matching slot exists within HTS probes
        for (int probe = 0; probe < HTS; probe++) {
            const int old = atomicCAS(&w.ht[slot].x, -1, key);
            if (old == -1 || old == key) break;
            slot = (slot + 1) & (HTS - 1);
        }
        atomicMin(&w.ht[slot].y, it);
        w.slot[it] = (short)slot;
    }
    __syncwarp();
    for (int it = lane; it < n; it += 32) {
        const bool dup = w.ht[w.slot[it]].y != it;
        bp[it].actidx = dup ? 1 : -1;   // marks: 1 = merge pending, -1 = alive, -2 = erased
        anydup |= dup;
    }
    __syncwarp();
    if (__any_sync(FULL, anydup) && lane == 0) {
        for (int it = 0; it < n; it++) {
            BPh &b = bp[it];
            if (b.actidx != 1) continue;
            int2 &hs = w.ht[w.slot[it]];
            BPh &o = bp[hs.y];
            if (o.prob > b.prob) {
                o.weight = __fadd_rn(o.weight, __fmul_rn(b.weight, __fdiv_rn(b.prob, o.prob)));
                b.actidx = -2;
            } else {
                b.weight = __fadd_rn(b.weight, __fmul_rn(o.weight, __fdiv_rn(o.prob, b.prob)));
                o.actidx = -2;
                b.actidx = -1;
                hs.y = it;
            }
        }
    }
    __syncwarp();
    BPh *dst = w.bp[w.bpsel ^ 1];
    int keep = 0;
    for (int base = 0; base < n; base += 32) {
        const int it = base + lane;
        const bool alive = it < n && bp[it].actidx != -2;
        const unsigned ba = __ballot_sync(FULL, alive);
        if (alive) {
            BPh &o = dst[keep + __popc(ba & lanemask_lt())];
            o = bp[it];
            o.actidx = -1;
        }
        keep += __popc(ba);
    }
    for (int it = lane; it < n; it += 32) w.ht[w.slot[it]] = make_int2(-1, INT_MAX);
    if (lane == 0) { w.nbp = keep; w.bpsel ^= 1; }
    __syncwarp();
}

// Beam::advanceBeamFront (Beam.cpp:263-539)
__device__ int beam_advance(const Ctx &c, WS &w) {
    const int lane = lane_id();
    // every lane has read the cursor for its loop condition before lane 0
    // moves it (otherwise lanes could leave the caller's loop at different
    // iterations and meet different warp collectives)
    __syncwarp();
    if (lane == 0) w.cursor += w.reverse ? -1 : 1;
    __syncwarp();
    beam_calc_rec(c, w);
    beam_load_rows(c, w);
    const int cursor = w.cursor;
    Cons cn = w.constr[cursor];
    while (true) {
        BPh *bp = w.bp[w.bpsel];
        const int nbp = w.nbp, nhap = w.nhap;
        // markRequiredExtensions (only sets flags: order free)
        for (int it = lane; it < nbp; it += 32) {
            hp_mark_required(c.hp[c.happ[bp[it].mat]], cn);
            hp_mark_required(c.hp[c.happ[bp[it].pat]], cn);
        }
        __syncwarp();
        // happath extensions, one path per lane
        int minse = 0, maxse = INT_MIN;
        for (int i = lane; i < nhap; i += 32) {
            const int id = c.happ[i];
            HPh &h = c.hp[id];
            if (h.toext0 || h.toext1) {
                const int se = hp_extend(c, w, id);
                if (se < minse) minse = se;
                if (se > maxse) maxse = se;
            }
        }
        for (int o = 16; o; o >>= 1) {
            minse = min(minse, __shfl_xor_sync(0xffffffffu, minse, o));
            maxse = max(maxse, __shfl_xor_sync(0xffffffffu, maxse, o));
        }
        const int bpscaleexp = -(maxse + minse);
        __syncwarp();
        // beam-path extensions
        float maxP = 0.0f;
        const int g = c.tg[cursor];
        for (int it = lane; it < nbp; it += 32) {
            const float mp = bp_extend(c, bp[it], g, cn, bpscaleexp);
            if (maxP < mp) maxP = mp;
        }
        for (int o = 16; o; o >>= 1) maxP = fmaxf(maxP, __shfl_xor_sync(0xffffffffu, maxP, o));
        __syncwarp();
        if (beam_prune_select(c, w, maxP, cn)) break;
        if (cn.type != C_NONE) { cn.type = C_NONE; continue; }
        if (lane == 0) w.err |= EIMP_ERR_BEAM_EMPTY;
        __syncwarp();
        return -1;
    }
    beam_apply_hap(c, w);
    if (w.err) return -1;
    beam_apply_bp(c, w);
    if (w.err) return -1;
    beam_merge(c, w);
    return 0;
}

// Beam::callKeepPhaseProb (Beam.cpp:95-185): the lanes classify the beam
// paths and prepare each path's terms of the two sums (0 where a path adds
// nothing, which leaves a float sum unchanged); lane 0 adds them in list order
__device__ float beam_call_keep(const Ctx &c, WS &w, int ci, int twoback) {
    const int lane = lane_id();
    if (lane == 0) {
        const int cl = c.calls[ci];
        const int front = w.reverse ? max(cl - w.Delta, 0) : min(cl + w.Delta, c.S - 1);
        w.curridx = w.reverse ? cl - front : front - cl;
        const int r = w.reverse ? (twoback ? c.calls[ci + 2] : c.calls[ci + 1])
                                : (twoback ? c.calls[ci - 2] : c.calls[ci - 1]);
        w.refidx = w.reverse ? r - front : front - r;
        w.ires = front;
    }
    __syncwarp();
    const int front = w.ires;
    while ((w.reverse && w.cursor > front) || (!w.reverse && w.cursor < front))
        if (beam_advance(c, w)) return -1.0f;
    const BPh *bp = w.bp[w.bpsel];
    const int n = w.nbp, curridx = w.curridx, refidx = w.refidx;
    for (int it = lane; it < n; it += 32) {
        const BPh &b = bp[it];
        const HPh &hm = c.hp[c.happ[b.mat]], &hq = c.hp[c.happ[b.pat]];
        const int cf = bh_at(hm, curridx), cs = bh_at(hq, curridx);
        const int rf = bh_at(hm, refidx), rs = bh_at(hq, refidx);
        const float p = __fmul_rn(b.weight, b.prob);
        float k, s;
        if (cf != cs && rf != rs) {
            k = cf == rf ? p : 0.0f;
            s = cf == rf ? 0.0f : p;
        } else {
            k = __fdiv_rn(p, 2.0f);
            s = k;
        }
        w.acc0[it] = k; w.acc1[it] = s;
    }
    __syncwarp();
    if (lane == 0) {
        float acckp = 0.0f, accsp = 0.0f;
        for (int it = 0; it < n; it++) { acckp = __fadd_rn(acckp, w.acc0[it]); accsp = __fadd_rn(accsp, w.acc1[it]); }
        float ret = 0.5f;
        if (__fadd_rn(acckp, accsp) > 0.0f) ret = __fdiv_rn(acckp, __fadd_rn(acckp, accsp));
        w.fres = ret;
    }
    __syncwarp();
    return w.fres;
}

// Beam::callDosage (Beam.cpp:187-261), split like beam_call_keep
__device__ float beam_call_dosage(const Ctx &c, WS &w, int si) {
    const int lane = lane_id();
    if (lane == 0) {
        const int front = w.reverse ? max(si - w.Delta, 0) : min(si + w.Delta, c.S - 1);
        w.curridx = w.reverse ? si - front : front - si;
        w.refidx = -1;
        w.ires = front;
    }
    __syncwarp();
    const int front = w.ires;
    while ((w.reverse && w.cursor > front) || (!w.reverse && w.cursor < front))
        if (beam_advance(c, w)) return -1.0f;
    const BPh *bp = w.bp[w.bpsel];
    const int n = w.nbp, curridx = w.curridx;
    for (int it = lane; it < n; it += 32) {
        const BPh &b = bp[it];
        const HPh &hm = c.hp[c.happ[b.mat]], &hq = c.hp[c.happ[b.pat]];
        const int cf = bh_at(hm, curridx), cs = bh_at(hq, curridx);
        const float p = __fmul_rn(b.weight, b.prob);
        w.acc0[it] = p;
        w.acc1[it] = cf == cs ? (cf == 1 ? __fmul_rn(2.0f, p) : 0.0f) : p;
    }
    __syncwarp();
    if (lane == 0) {
        float dos = 0.0f, ptot = 0.0f;
        for (int it = 0; it < n; it++) { ptot = __fadd_rn(ptot, w.acc0[it]); dos = __fadd_rn(dos, w.acc1[it]); }
        float ret = 1.0f;
        if (ptot > 0.0f) ret = __fdiv_rn(dos, ptot);
        w.fres = ret;
    }
    __syncwarp();
    return w.fres;
}

__host__ __device__ __forceinline__ size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace


// arena layout per target (bytes)
struct ArenaLayout {
    size_t hp, ph, ivpool, ivfree, happ, happ_old, hapmap, fstack, copies, heap, cons, rcons, probs, confs, tg, total;
    int NH, HMAX;
};

static ArenaLayout arena_layout(const BeamParams &p, int M) {
    ArenaLayout a;
    int P = p.P > p.Pf ? p.P : p.Pf;
    int H = p.H > p.Hf ? p.H : p.Hf;
    a.NH = 4 * P + 8;
    a.HMAX = H;
    size_t o = 0;
    a.hp = o; o = align256(o + sizeof(HPh) * a.NH);
    a.ph = o; o = align256(o + sizeof(float) * PHMAX * a.NH);
    // the interval pool doubles as the storage of the pre-phasing constraint
    // heaps (one entry per split site) once the fast beam is done
    const size_t ivb = sizeof(uint32_t) * (size_t)H * 3 * a.NH, heapb = sizeof(Hel) * (size_t)(M + 1);
    a.ivpool = o; o = align256(o + (ivb > heapb ? ivb : heapb));
    a.ivfree = o; o = align256(o + sizeof(int) * 3 * a.NH);
    a.happ = o; o = align256(o + sizeof(int) * a.NH);
    a.happ_old = o; o = align256(o + sizeof(int) * a.NH);
    a.hapmap = o; o = align256(o + sizeof(int2) * a.NH);
    a.fstack = o; o = align256(o + sizeof(int) * a.NH);
    a.copies = o; o = align256(o + sizeof(int) * 3 * a.NH);
    a.heap = o; o = align256(o + sizeof(Hel) * (PMAX + 2));
    a.cons = o; o = align256(o + sizeof(Cons) * (size_t)(M + 1));
    a.rcons = o; o = align256(o + sizeof(Cons) * (size_t)(M + 1));
    a.probs = o; o = align256(o + sizeof(float) * (size_t)(M + 1));
    a.confs = o; o = align256(o + sizeof(float) * (size_t)(M + 1));
    a.tg = o; o = align256(o + (size_t)(M + 1));
    a.total = o;
    return a;
}

size_t beam_arena_bytes(const BeamParams &p, int M) { return arena_layout(p, M).total; }

// shared memory per warp besides its WS: the cursor's two PBWT rows and the
// merge key of each haplotype path
__host__ __device__ __forceinline__ size_t beam_rows_bytes(int K) { return ((2 * eimp_kw(K) * 4 + 15) / 16) * 16; }
__host__ __device__ __forceinline__ size_t beam_canon_bytes(int NH) { return (((size_t)NH * 2 + 15) / 16) * 16; }

__device__ __forceinline__ void setbit_(uint64_t *v, int i) { v[i >> 6] |= 1ull << (i & 63); }
__device__ __forceinline__ void clrbit_(uint64_t *v, int i) { v[i >> 6] &= ~(1ull << (i & 63)); }

// Targets in longest-first order: order[rank] = target, ranked by split sites
// descending, ties by index.  One CTA; the persistent beam below takes the
// targets in this order, so the longest walks start first and the short ones
// fill the end of the launch.
__global__ void lpt_order_kernel(const int32_t *__restrict__ nsplits, int ntgt, int32_t *__restrict__ order,
                                 const int *__restrict__ skip) {
    if (skip && *skip) return;
    for (int i = threadIdx.x; i < ntgt; i += blockDim.x) {
        const int si = nsplits[i];
        int rank = 0;
        for (int j = 0; j < ntgt; j++) {
            const int sj = nsplits[j];
            rank += sj > si || (sj == si && j < i);
        }
        order[rank] = i;
    }
}

// Target::phaseExtPBWT (Target.cpp:291-777), one warp per target.  The grid
// is persistent (as many CTAs as are resident at once): every warp takes the
// next target from a device counter, in the order given (longest first), and
// phases it with the beam arena of its slot, so the arenas number the
// resident warps, not the targets.
// The persistent beam, WARPS targets (warps) per CTA (the kernel below).
template <int WARPS>
__device__ __forceinline__ void beam_run(
    const BeamParams &p, const ArenaLayout &al, int ntgt, int M, const uint8_t *__restrict__ gt, const uint64_t *__restrict__ monos,
    const int32_t *__restrict__ splits, const int32_t *__restrict__ nsplits, const int32_t *__restrict__ calls,
    const int32_t *__restrict__ ncalls, const float *__restrict__ cmdiffs, const uint32_t *__restrict__ pbwt,
    const int32_t *__restrict__ count0, const int64_t *__restrict__ rowoff, uint8_t *__restrict__ arena,
    size_t arena_bytes, uint64_t *__restrict__ mats, uint64_t *__restrict__ pats, float *__restrict__ dmat,
    float *__restrict__ dpat, float *__restrict__ totalconf, int32_t *__restrict__ ncallsites,
    uint32_t *__restrict__ status, const int *__restrict__ skip, const int32_t *__restrict__ order,
    int *__restrict__ workq) {
    if (skip && *skip) return;   // the batch exceeds the reserved rows
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WS &w = reinterpret_cast<WS *>(smem_raw)[wid];
    uint8_t *const ab = arena + (size_t)(blockIdx.x * WARPS + wid) * arena_bytes;
    for (;;) {
    int qi = 0;
    if (lane == 0) qi = atomicAdd(workq, 1);
    qi = __shfl_sync(0xffffffffu, qi, 0);
    if (qi >= ntgt) break;
    const int t = order[qi];
    const int wM = (int)eimp_W(M);
    const uint8_t *g = gt + (size_t)t * M;
    const uint64_t *mo = monos + (size_t)t * wM;
    uint64_t *mat = mats + (size_t)t * wM;
    uint64_t *pat = pats + (size_t)t * wM;
    float *dm = dmat + (size_t)t * M;
    float *dp = dpat + (size_t)t * M;
    for (int i = lane; i < wM; i += 32) { mat[i] = 0ull; pat[i] = 0ull; }
    for (int i = lane; i < M; i += 32) { dm[i] = 0.0f; dp[i] = 0.0f; }

    const int S = nsplits[t];
    const int C = ncalls[t];
    const int K = p.K;
    const size_t kw = eimp_kw(K);
    if (lane == 0) {   // the warp's PBWT row pair and merge keys after the WS array
        uint8_t *base = smem_raw + sizeof(WS) * WARPS;
        w.rowinc = reinterpret_cast<uint32_t *>(base + (size_t)wid * beam_rows_bytes(K));
        w.rowref = w.rowinc + kw;
        w.canon = reinterpret_cast<short *>(base + (size_t)WARPS * beam_rows_bytes(K) +
                                            (size_t)wid * beam_canon_bytes(al.NH));
        w.heap = reinterpret_cast<Hel *>(ab + al.heap);
    }
    Ctx c;
    c.hp = reinterpret_cast<HPh *>(ab + al.hp);
    c.ph = reinterpret_cast<float *>(ab + al.ph);
    c.ivpool = reinterpret_cast<uint32_t *>(ab + al.ivpool);
    c.ivfree = reinterpret_cast<int *>(ab + al.ivfree);
    c.happ = reinterpret_cast<int *>(ab + al.happ);
    c.happ_old = reinterpret_cast<int *>(ab + al.happ_old);
    c.hapmap = reinterpret_cast<int2 *>(ab + al.hapmap);
    c.fstack = reinterpret_cast<int *>(ab + al.fstack);
    c.copies = reinterpret_cast<int *>(ab + al.copies);
    c.NH = al.NH; c.HMAX = al.HMAX;
    Cons *cons = reinterpret_cast<Cons *>(ab + al.cons);
    Cons *rcons = reinterpret_cast<Cons *>(ab + al.rcons);
    float *phaseProbs = reinterpret_cast<float *>(ab + al.probs);
    float *callConfs = reinterpret_cast<float *>(ab + al.confs);
    uint8_t *tg = ab + al.tg;
    const int64_t r0 = rowoff[t];
    c.Mp = 2 * S + 1;
    c.rows = pbwt + (size_t)2 * r0 * kw;
    c.count0 = count0 + r0;
    c.K = K; c.kw = (int)kw;
    c.Kinv = (float)(1.0 / (double)(float)K);
    c.cmd = cmdiffs + (size_t)t * (M + 1);
    c.S = S;
    c.calls = calls + (size_t)t * M;
    c.ncalls = C;
    c.tg = tg;
    c.pErr = p.pErr; c.pLimit = p.pLimit; c.expectIBDcM = p.expectIBDcM;
    const int32_t *sp = splits + (size_t)t * M;
    for (int s = lane; s < S; s += 32) { tg[s] = g[sp[s]]; cons[s].type = C_NONE; cons[s].refidx = 0; }
    __syncwarp();

    int err = 0;
    const int startph = p.startph ? (p.startph[t] != 0) : 0;   // VCFData::getStartPhase (Target.cpp:311-312)
    int cur = startph, lastph = startph;
    if (p.doPrePhasing) {   // Target.cpp:324-438
        beam_init(c, w, cons, 0, p.Hf, p.Pf, p.Deltaf);
        if (lane == 0 && S > 0) { cons[0].type = C_HETKEEP; cons[0].refidx = 0; }
        __syncwarp();
        int nci = 1;
        for (int si = 1; si < S && !err; si++) {
            if (si == c.calls[nci]) {
                float pr = (float)((double)beam_call_keep(c, w, nci, 0) - 0.5);
                if (w.err) { err = 1; break; }
                int ref = cur;
                int refidx = c.calls[nci] - c.calls[nci - 1] - 1;
                if (nci > 1) {
                    float p2 = (float)((double)beam_call_keep(c, w, nci, 1) - 0.5);
                    if (w.err) { err = 1; break; }
                    if (fabsf(p2) > fabsf(pr)) { pr = p2; ref = lastph; refidx = c.calls[nci] - c.calls[nci - 2] - 1; }
                }
                lastph = cur;
                int type;
                if (pr < 0.0f) { cur = !ref; type = C_HETSWITCH; } else { cur = ref; type = C_HETKEEP; }
                if (lane == 0) { cons[si].type = type; cons[si].refidx = refidx; phaseProbs[si] = fabsf(pr); }
                nci++;
            } else {
                float pr = beam_call_dosage(c, w, si);
                if (w.err) { err = 1; break; }
                if (lane == 0) {
                    if (tg[si] == 0) { cons[si].type = C_HOMREF; cons[si].refidx = 0; pr = (float)(2.0 - (double)pr); }
                    else { cons[si].type = C_HOMALT; cons[si].refidx = 0; }
                    phaseProbs[si] = pr;
                }
            }
            __syncwarp();
        }
        if (!err && lane == 0) {
            // the constraint heaps (Target.cpp:402-436), filled in site order as
            // the reference does; the interval pool of the finished fast beam
            // serves as heap storage
            Hel *hq = reinterpret_cast<Hel *>(c.ivpool);
            for (int pass = 0; pass < 2; pass++) {   // 0: call sites, 1: homozygous split sites
                int n = 0;
                int nci2 = 1;
                for (int si = 1; si < S; si++) {
                    bool iscall = (si == c.calls[nci2]);
                    if (iscall) nci2++;
                    if ((pass == 0) == iscall) heap_push(hq, n, phaseProbs[si], si, 0);
                }
                const size_t total = (size_t)n;
                const size_t smin = (size_t)__fmul_rn((float)total, p.minfixsize);
                const size_t smax = (size_t)((double)total * (1.0 - (double)p.maxfixsize));
                size_t si;
                const double thrmax = pass == 0 ? (double)p.maxfixthr - 0.5 : (double)p.maxfixthr * 2.0;
                const double thrmin = pass == 0 ? (double)p.minfixthr - 0.5 : (double)p.minfixthr * 2.0;
                for (si = 0; si < smin; si++) {
                    Hel cc = heap_popmin(hq, n);
                    if ((double)cc.key >= thrmax || ((double)cc.key >= thrmin && si >= smax)) break;
                    cons[cc.a].type = C_NONE;
                }
                if (pass == 0 && si == smin) {
                    // (Target.cpp:416-425: compared against the shrinking heap)
                    for (; si < (size_t)n; si++) {
                        Hel cc = heap_popmin(hq, n);
                        if (cc.key > 0.0f) break;
                        cons[cc.a].type = C_NONE;
                    }
                }
            }
        }
        __syncwarp();
    }

    // fine phasing forward (Target.cpp:458-599)
    cur = startph;   // Target.cpp:443
    int nprobs = 0;
    if (lane == 0) phaseProbs[0] = 0.0f;
    nprobs = 1;
    if (!err) {
        beam_init(c, w, cons, 0, p.H, p.P, p.Delta);
        int m = 0;
        const int stop = S > 0 ? sp[c.calls[0]] : M;
        if (lane == 0) {
            for (; m < stop; m++) {
                uint8_t gg = g[m];
                if (gg == 2) { setbit_(mat, m); setbit_(pat, m); dm[m] = 1.0f; dp[m] = 1.0f; }
                else if (gg == 1) { setbit_(pat, m); dm[m] = 0.5f; dp[m] = 0.5f; }
            }
            if (m < M) { if (cur) setbit_(mat, m); else setbit_(pat, m); }
        }
        m = stop;
        if (m < M) m++;
        int nci = 1;
        for (; m < M && !err; m++) {
            const uint8_t gg = g[m];
            if (gg == 1) {
                const bool mono = (mo[m >> 6] >> (m & 63)) & 1ull;
                if (!mono) {
                    float pr = (float)((double)beam_call_keep(c, w, nci, 0) - 0.5);
                    if (w.err) { err = 1; break; }
                    if (lane == 0) phaseProbs[nprobs] = pr;
                    nprobs++;
                    cur = pr < 0.0f ? !cur : cur;
                    nci++;
                } else if (lane == 0) { dm[m] = 0.5f; dp[m] = 0.5f; }
                if (lane == 0) { if (cur) setbit_(mat, m); else setbit_(pat, m); }
            } else if (gg == 2 && lane == 0) {
                setbit_(mat, m); setbit_(pat, m); dm[m] = 1.0f; dp[m] = 1.0f;
            }
        }
        __syncwarp();
    }
    if (!err && S > 0) {   // Target.cpp:601-619
        if (lane == 0) {
            for (int i = 0; i < C; i++) callConfs[i] = 0.0f;
            if (p.doRevPhasing) callConfs[C - 1] = (float)((double)fabsf(phaseProbs[nprobs - 1]) + 0.5);
            else for (int i = 0; i < nprobs && i < C; i++) callConfs[i] = (float)((double)fabsf(phaseProbs[i]) + 0.5);
        }
        __syncwarp();
    }
    if (!err && p.doRevPhasing && S > 0) {   // Target.cpp:620-758
        if (lane == 0) {
            for (int s = 0; s < S; s++) { rcons[s].type = C_NONE; rcons[s].refidx = 0; }
            for (int ci = 1; ci < S; ci++) {
                Cons cc = cons[ci];
                if (cc.type == C_HETKEEP || cc.type == C_HETSWITCH) {
                    Cons &r = rcons[ci - cc.refidx - 1];
                    if (r.type != C_NONE) {
                        int ridx = ci - cc.refidx + r.refidx;
                        rcons[ridx].refidx = cc.refidx - r.refidx - 1;
                        rcons[ridx].type = (cc.type != r.type) ? C_HETSWITCH : C_HETKEEP;
                    } else { r.type = cc.type; r.refidx = cc.refidx; }
                } else if (cc.type == C_HOMREF || cc.type == C_HOMALT) {
                    rcons[ci].type = cc.type;
                }
            }
            rcons[S - 1].type = C_HETKEEP; rcons[S - 1].refidx = 0;
            float last = phaseProbs[nprobs - 1];
            float dref = last < 0.0f ? (float)(0.5 + (double)last) : (float)(0.5 - (double)last);
            float dalt = last < 0.0f ? (float)(0.5 - (double)last) : (float)(0.5 + (double)last);
            int site = sp[c.calls[C - 1]];
            dm[site] = cur == 0 ? dref : dalt;
            dp[site] = cur == 0 ? dalt : dref;
        }
        __syncwarp();
        beam_init(c, w, rcons, 1, p.H, p.P, p.Delta);
        for (int rci = C - 2; rci >= 0 && !err; rci--) {
            float pr = (float)((double)beam_call_keep(c, w, rci, 0) - 0.5);
            if (w.err) { err = 1; break; }
            float fw = phaseProbs[rci + 1];
            if (fabsf(fw) > fabsf(pr)) pr = fw;
            cur = pr < 0.0f ? !cur : cur;
            if (lane == 0) {
                int s2 = sp[c.calls[rci]];
                if (cur) { setbit_(mat, s2); clrbit_(pat, s2); } else { clrbit_(mat, s2); setbit_(pat, s2); }
                float dref = pr < 0.0f ? (float)(0.5 + (double)pr) : (float)(0.5 - (double)pr);
                float dalt = pr < 0.0f ? (float)(0.5 - (double)pr) : (float)(0.5 + (double)pr);
                dm[s2] = cur == 0 ? dref : dalt;
                dp[s2] = cur == 0 ? dalt : dref;
                callConfs[rci] = (float)((double)fabsf(pr) + 0.5);
            }
            __syncwarp();
        }
    }
    if (lane == 0) {
        float tc = 0.0f;
        int nc = 0;
        if (!err && S > 0) {   // Target.cpp:761-772
            for (int i = 0; i < C; i++) tc = __fadd_rn(tc, callConfs[i]);
            nc = C;
        }
        totalconf[t] = tc;
        ncallsites[t] = nc;
        if (err) atomicOr(status, w.err ? w.err : (uint32_t)EIMP_ERR_BEAM_EMPTY);
    }
    __syncwarp();
    }
}

__global__ void __launch_bounds__(32 * BEAM_WARPS, 1) beam_kernel(
    BeamParams p, ArenaLayout al, int ntgt, int M, const uint8_t *__restrict__ gt, const uint64_t *__restrict__ monos,
    const int32_t *__restrict__ splits, const int32_t *__restrict__ nsplits, const int32_t *__restrict__ calls,
    const int32_t *__restrict__ ncalls, const float *__restrict__ cmdiffs, const uint32_t *__restrict__ pbwt,
    const int32_t *__restrict__ count0, const int64_t *__restrict__ rowoff, uint8_t *__restrict__ arena,
    size_t arena_bytes, uint64_t *__restrict__ mats, uint64_t *__restrict__ pats, float *__restrict__ dmat,
    float *__restrict__ dpat, float *__restrict__ totalconf, int32_t *__restrict__ ncallsites,
    uint32_t *__restrict__ status, const int *__restrict__ skip, const int32_t *__restrict__ order,
    int *__restrict__ workq) {
    beam_run<BEAM_WARPS>(p, al, ntgt, M, gt, monos, splits, nsplits, calls, ncalls, cmdiffs, pbwt, count0, rowoff, arena, arena_bytes, mats,
                      pats, dmat, dpat, totalconf, ncallsites, status, skip, order, workq);
}

static size_t beam_smem(const BeamParams &p, const ArenaLayout &al, int warps) {
    return (sizeof(WS) + beam_rows_bytes(p.K) + beam_canon_bytes(al.NH)) * warps;
}

int beam_slots(const BeamParams &p, int M, int ntgt, int pct) {
    const ArenaLayout al = arena_layout(p, M);
    const size_t sm = beam_smem(p, al, BEAM_WARPS);
    int dev = 0, nsm = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -1;
    if (ensure_dynamic_smem((const void *)beam_kernel, sm) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, beam_kernel, 32 * BEAM_WARPS, sm) != cudaSuccess || per < 1)
        return -1;
    int ctas = (int)((long)per * nsm * (pct < 1 ? 1 : pct > 100 ? 100 : pct) / 100);
    if (ctas < 1) ctas = 1;
    const int need = (ntgt + BEAM_WARPS - 1) / BEAM_WARPS;
    return (need < ctas ? need : ctas) * BEAM_WARPS;
}

cudaError_t launch_beam(const BeamParams &p, int ntgt, int M, const uint8_t *gt, const uint64_t *monos,
                        const int32_t *splits, const int32_t *nsplits, const int32_t *calls, const int32_t *ncalls,
                        const float *cmdiffs, const uint32_t *pbwt, const int32_t *count0, const int64_t *rowoff,
                        void *arena, size_t arena_bytes, int slots, int32_t *order, int *workq, uint64_t *mats,
                        uint64_t *pats, float *dmat, float *dpat, float *totalconf, int32_t *ncallsites,
                        uint32_t *status, const int *skip, cudaStream_t st) {
    ArenaLayout al = arena_layout(p, M);
    if (arena_bytes < al.total || slots < BEAM_WARPS || slots % BEAM_WARPS) return cudaErrorInvalidValue;
    const size_t sm = beam_smem(p, al, BEAM_WARPS);
    cudaError_t e = ensure_dynamic_smem((const void *)beam_kernel, sm);
    if (e != cudaSuccess) return e;
    lpt_order_kernel<<<1, 1024, 0, st>>>(nsplits, ntgt, order, skip);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(workq, 0, sizeof(int), st)) != cudaSuccess) return e;
    beam_kernel<<<slots / BEAM_WARPS, 32 * BEAM_WARPS, sm, st>>>(p, al, ntgt, M, gt, monos, splits, nsplits, calls,
                                                                ncalls, cmdiffs, pbwt, count0, rowoff,
                                                                (uint8_t *)arena, arena_bytes, mats, pats, dmat, dpat,
                                                                totalconf, ncallsites, status, skip, order, workq);
    return cudaGetLastError();
}

}  // namespace eimp
