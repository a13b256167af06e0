// PBWT imputation kernels for B200 (sm_100a).
//
//  refpbwt_kernel   -- PBWT::buildComprPBWT with refPBWT=true (PBWT.cpp:207-285,
//                      136-142): compressed rows + prefix arrays gAbsPerm.
//  transpose_kernel -- site-major -> haplotype-major bit matrix (64x64 tiles).
//  smm_kernel       -- TargetImp::calcSMMatches / processHistorySubTree
//                      (TargetImp.cpp:74-246, 346-435), one warp per target
//                      haplotype: the rank queries of all tree nodes of a site
//                      run across the lanes, the tree update runs on lane 0.
//  dosage_kernel    -- TargetImp::imputeBunch (TargetImp.cpp:474-558), one
//                      warp per (target haplotype, 64-site tile).
#include "common.cuh"
#include "kernels.h"

namespace eimp {

// ---------------------------------------------------------------------------
// block-wide exclusive scan of an int array in shared memory (length n)
// ---------------------------------------------------------------------------
__device__ void block_exscan(int *a, int n, int *warpbuf, int *total) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per = (n + nt - 1) / nt;
    const int lo = tid * per, hi = min(n, lo + per);
    int s = 0;
    for (int i = lo; i < hi; i++) s += a[i];
    // inclusive scan of s across the block
    int lane = tid & 31, wid = tid >> 5;
    int v = s;
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warpbuf[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int nw = (nt + 31) >> 5;
        int w = lane < nw ? warpbuf[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) warpbuf[lane] = w;
    }
    __syncthreads();
    int excl = v - s + (wid ? warpbuf[wid - 1] : 0);
    for (int i = lo; i < hi; i++) { int t = a[i]; a[i] = excl; excl += t; }
    if (total && tid == nt - 1) *total = excl;
    __syncthreads();
}

// ---------------------------------------------------------------------------
// reference PBWT with prefix arrays.  One CTA sweeps the M sites in order;
// absperm[m] is the order before site m, absperm[m+1] is written from it.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) refpbwt_kernel(const uint64_t *__restrict__ sitemajor, int M, int K,
                                                      int wN, uint32_t *__restrict__ compr,
                                                      int32_t *__restrict__ absperm, int32_t *__restrict__ count0) {
    extern __shared__ uint8_t smem[];
    const int nwords = (K + 31) / 32;
    uint32_t *row = reinterpret_cast<uint32_t *>(smem);                  // 2*wN u32
    uint32_t *data = row + 2 * wN;                                       // nwords
    int *pz = reinterpret_cast<int *>(data + nwords);                    // nwords + 1
    int *warpbuf = pz + nwords + 1;                                      // 32
    int *tot = warpbuf + 32;                                             // 1
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
    const size_t kw = 2 * (size_t)nwords;

    for (int i = tid; i < K; i += blockDim.x) absperm[i] = i;
    __syncthreads();
    for (int m = 0; m < M; m++) {
        const uint64_t *src = sitemajor + (size_t)m * wN;
        for (int w = tid; w < wN; w += blockDim.x) {
            uint64_t x = src[w];
            row[2 * w] = (uint32_t)x;
            row[2 * w + 1] = (uint32_t)(x >> 32);
        }
        __syncthreads();
        const int32_t *perm = absperm + (size_t)m * K;
        int32_t *nperm = absperm + (size_t)(m + 1) * K;
        // pass 1: bits in prefix order, zeros per 32-position word
        for (int w = wid; w < nwords; w += nwarps) {
            int i = w * 32 + lane;
            int bit = 1;
            if (i < K) {
                int h = perm[i];
                bit = (row[h >> 5] >> (h & 31)) & 1;
            }
            uint32_t b = __ballot_sync(0xffffffffu, bit);
            if (lane == 0) { data[w] = b; pz[w] = __popc(~b); }
        }
        __syncthreads();
        block_exscan(pz, nwords, warpbuf, tot);
        const int cnt0 = *tot;
        // pass 2: scatter into the next order, emit compressed words
        uint32_t *crow = compr + (size_t)m * kw;
        for (int w = wid; w < nwords; w += nwarps) {
            int i = w * 32 + lane;
            uint32_t b = data[w];
            int zb = pz[w];
            if (i < K) {
                int h = perm[i];
                uint32_t lt = (1u << lane) - 1u;
                int dst = ((b >> lane) & 1) ? cnt0 + (w * 32 - zb) + __popc(b & lt) : zb + __popc(~b & lt);
                nperm[dst] = h;
            }
            if (lane == 0) {
                crow[2 * w] = b;
                crow[2 * w + 1] = (uint32_t)(zb + __popc(~b));
            }
        }
        if (tid == 0) count0[m] = cnt0;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// bit-matrix transpose: src (rows x srcw words, 'cols' valid bits per row) ->
// dst (cols x dstw words).  One 64x64 tile per block of 64 threads.
// ---------------------------------------------------------------------------
__global__ void transpose_kernel(const uint64_t *__restrict__ src, size_t rows, size_t srcw,
                                 uint64_t *__restrict__ dst, size_t cols, size_t dstw) {
    __shared__ uint64_t tile[64];
    const size_t rw = blockIdx.x;      // 64-row block (source rows -> dest word)
    const size_t cw = blockIdx.y;      // source word (-> 64 dest rows)
    const int t = threadIdx.x;
    size_t r = rw * 64 + t;
    tile[t] = (r < rows && cw < srcw) ? src[r * srcw + cw] : 0ull;
    __syncthreads();
    size_t c = cw * 64 + t;
    if (c < cols && rw < dstw) {
        uint64_t o = 0;
#pragma unroll 8
        for (int j = 0; j < 64; j++) o |= ((tile[j] >> t) & 1ull) << j;
        dst[c * dstw + rw] = o;
    }
}

// ---------------------------------------------------------------------------
// set-maximal matches
//
// The history tree of TargetImp::processHistorySubTree lives in shared memory,
// one pool per warp.  Per site: lane 0 lists the live nodes in pre-order, all
// lanes map their intervals through the site's PBWT row in parallel (the
// mapping of a node depends only on its own interval, and a node's interval is
// not changed before the recursion reaches it), then lane 0 replays the
// recursion iteratively with the precomputed mappings.
// ---------------------------------------------------------------------------
struct SmmNode {
    int l, r;
    int de;              // depth | errors << 24
    short left, right;   // node indices, -1 = none
};
struct SmmFrame {
    short lt, rt;        // slots (see slot encoding)
    int cdepth;          // max depth returned by the children
    unsigned char st;    // bits: 0-1 stage, 2 perase, 3 extend0, 4 extend1
};

// slot encoding: s >= 0 -> node (s>>1).left (s&1==0) or .right (s&1==1);
// SLOT_ROOT -> the root variable
#define SLOT_ROOT (-2)

struct SmmWarpSmem {
    SmmNode node[SMM_NODES];
    int4 map[SMM_NODES];
    SmmFrame stack[SMM_NODES];
    short order[SMM_NODES];
    short freel[SMM_NODES];
};

__device__ __forceinline__ short &slot_ref(SmmWarpSmem &S, short &rootvar, int s) {
    if (s == SLOT_ROOT) return rootvar;
    return (s & 1) ? S.node[s >> 1].right : S.node[s >> 1].left;
}
__device__ __forceinline__ int de_depth(int de) { return de & 0xffffff; }
__device__ __forceinline__ int de_err(int de) { return (int)((unsigned)de >> 24); }

__global__ void __launch_bounds__(SMM_WARPS * 32) smm_kernel(
    const uint32_t *__restrict__ compr, const int32_t *__restrict__ count0, int M, int K,
    const uint64_t *__restrict__ phased, int wM, const uint8_t *__restrict__ gt, int nhaps,
    int setmaxerrors, int4 *__restrict__ matches, int cap, int *__restrict__ nmatch,
    uint32_t *__restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int hap = blockIdx.x * SMM_WARPS + wid;
    if (hap >= nhaps) return;
    SmmWarpSmem &S = reinterpret_cast<SmmWarpSmem *>(smem_raw)[wid];
    const uint8_t *g = gt + (size_t)(hap >> 1) * M;
    const uint64_t *hw = phased + (size_t)hap * wM;
    int4 *out = matches + (size_t)hap * cap;
    const size_t kw = eimp_kw(K);

    // missingness > 50 %: no matches (TargetImp.cpp:79-80)
    int nmiss = 0;
    for (int m = lane; m < M; m += 32) nmiss += g[m] == 3;
    for (int o = 16; o; o >>= 1) nmiss += __shfl_xor_sync(0xffffffffu, nmiss, o);
    if (nmiss > M / 2) { if (lane == 0) nmatch[hap] = 0; return; }

    int nfree = 0, used = 0;
    short root = -1;
    int nres = 0, treedepth = 0;
    uint32_t err = 0;

    auto pool_new = [&](int l, int r, int de) -> int {
        int i;
        if (nfree) i = S.freel[--nfree];
        else if (used < SMM_NODES) i = used++;
        else { err |= EIMP_ERR_NODE_OVERFLOW; return -1; }
        SmmNode &n = S.node[i];
        n.left = -1; n.right = -1; n.l = l; n.r = r; n.de = de;
        return i;
    };
    auto pool_del = [&](int i) { S.freel[nfree++] = (short)i; };
    auto merge_single = [&](short &slot) {
        // TargetImp.cpp:405-415: a node with one child of equal mapping is
        // replaced by that child
        SmmNode &N = S.node[slot];
        if (N.left >= 0 && N.right < 0) {
            const SmmNode &C = S.node[N.left];
            if (C.l == N.l && C.r == N.r && de_err(C.de) == de_err(N.de)) { int t = slot; slot = N.left; pool_del(t); }
        } else if (N.left < 0 && N.right >= 0) {
            const SmmNode &C = S.node[N.right];
            if (C.l == N.l && C.r == N.r && de_err(C.de) == de_err(N.de)) { int t = slot; slot = N.right; pool_del(t); }
        }
    };

    // TargetImp.cpp:346-435 as an explicit-stack traversal (lane 0)
    auto process = [&](int lt0, int rt0, bool perase0, int m, int curr, int missing, int &newcount) -> int {
        int sp = 0;
        S.stack[0].lt = (short)lt0; S.stack[0].rt = (short)rt0; S.stack[0].cdepth = 0;
        S.stack[0].st = perase0 ? 4 : 0;
        int ret = 0;
        while (sp >= 0) {
            SmmFrame &f = S.stack[sp];
            int stage = f.st & 3;
            if (stage == 0) {
                int L = slot_ref(S, root, f.lt);
                bool perase = f.st & 4;
                int4 mp = perase ? make_int4(0, -1, 0, -1) : S.map[L];
                SmmNode &N = S.node[L];
                int ne = de_err(N.de);
                bool e0 = mp.x <= mp.y && (missing || !curr || ne < setmaxerrors);
                bool e1 = mp.z <= mp.w && (missing || curr || ne < setmaxerrors);
                if (e1) {
                    int ni = pool_new(mp.z, mp.w, (de_depth(N.de) + 1) | (((curr || missing) ? ne : ne + 1) << 24));
                    if (ni < 0) return -1;
                    slot_ref(S, root, f.rt) = (short)ni;
                }
                if (e0) {
                    N.l = mp.x; N.r = mp.y;
                    N.de = (de_depth(N.de) + 1) | (((curr && !missing) ? ne + 1 : ne) << 24);
                }
                if (!e0 && !e1) {
                    int d = de_depth(N.de);
                    if (d == treedepth && treedepth > 0) {
                        if (nres + newcount < cap) out[nres + newcount] = make_int4(m - d, m, N.l, N.r);
                        else err |= EIMP_ERR_MATCH_OVERFLOW;
                        newcount++;
                    }
                }
                unsigned char st = (unsigned char)(1 | (perase ? 4 : 0) | (e0 ? 8 : 0) | (e1 ? 16 : 0));
                f.st = st;
                if (N.left >= 0) {
                    if (sp + 1 >= SMM_NODES) { err |= EIMP_ERR_STACK_OVERFLOW; return -1; }
                    int R = slot_ref(S, root, f.rt);
                    SmmFrame &c = S.stack[++sp];
                    c.lt = (short)(2 * L); c.rt = (short)((R >= 0) ? 2 * R : f.rt);
                    c.cdepth = 0; c.st = (!e0 && !e1) ? 4 : 0;
                    continue;
                }
                stage = 1;
            }
            if (stage == 1) {
                f.st = (f.st & ~3) | 2;
                int L = slot_ref(S, root, f.lt);
                if (S.node[L].right >= 0) {
                    if (sp + 1 >= SMM_NODES) { err |= EIMP_ERR_STACK_OVERFLOW; return -1; }
                    int R = slot_ref(S, root, f.rt);
                    bool ce = !(f.st & 8) && !(f.st & 16);
                    SmmFrame &c = S.stack[++sp];
                    c.lt = (short)(2 * L + 1); c.rt = (short)((R >= 0) ? 2 * R + 1 : f.rt);
                    c.cdepth = 0; c.st = ce ? 4 : 0;
                    continue;
                }
            }
            // post-processing (TargetImp.cpp:392-432)
            int depth = f.cdepth;
            short &Ls = slot_ref(S, root, f.lt);
            if (f.st & 8) {
                int d = de_depth(S.node[Ls].de);
                if (d > depth) depth = d;
                merge_single(Ls);
            } else {
                pool_del(Ls);
                Ls = -1;
            }
            if (f.st & 16) {
                short &Rs = slot_ref(S, root, f.rt);
                int d = de_depth(S.node[Rs].de);
                if (d > depth) depth = d;
                merge_single(Rs);
            }
            sp--;
            if (sp >= 0) { if (depth > S.stack[sp].cdepth) S.stack[sp].cdepth = depth; }
            else ret = depth;
        }
        return ret;
    };

    if (lane == 0) root = (short)pool_new(0, K - 1, 0);
    bool failed = false;
    for (int m = 0; m < M && !failed; m++) {
        const int curr = bit_at(hw, m);
        const int missing = g[m] == 3;
        // pre-order of the tree below the (old) root; S.stack doubles as the
        // traversal stack (it is free between sites)
        int n = 0;
        if (lane == 0) {
            short *st = reinterpret_cast<short *>(S.stack);
            int sp = 0;
            st[sp++] = root;
            while (sp) {
                int x = st[--sp];
                S.order[n++] = (short)x;
                if (S.node[x].right >= 0) st[sp++] = S.node[x].right;
                if (S.node[x].left >= 0) st[sp++] = S.node[x].left;
            }
        }
        n = __shfl_sync(0xffffffffu, n, 0);
        __syncwarp();
        const uint32_t *crow = compr + (size_t)m * kw;
        const int c0 = count0[m];
        for (int i = lane; i < n; i += 32) {
            int x = S.order[i];
            int l0, r0, l1, r1;
            pbwt_map(crow, c0, S.node[x].l, S.node[x].r, l0, r0, l1, r1);
            S.map[x] = make_int4(l0, r0, l1, r1);
        }
        __syncwarp();
        if (lane == 0) {
            int nr = pool_new(0, K - 1, 0);
            if (nr < 0) failed = true;
            else {
                S.node[nr].left = root;
                root = (short)nr;
                int newcount = 0;
                int td = process(2 * root, 2 * root + 1, false, m, curr, missing, newcount);
                if (td < 0) failed = true;
                else {
                    // TargetImp.cpp:132-136: report only if no longer path is alive
                    if (newcount && nres < cap && out[nres].y - out[nres].x >= td && nres + newcount <= cap)
                        nres += newcount;
                    treedepth = td;
                }
            }
        }
        failed = __shfl_sync(0xffffffffu, (int)failed, 0);
        __syncwarp();
    }
    if (lane == 0) {
        if (!failed) {
            int newcount = 0;
            int td = process(SLOT_ROOT, SLOT_ROOT, true, M, 0, 0, newcount);
            if (td >= 0 && nres + newcount <= cap) nres += newcount;
        }
        nmatch[hap] = err ? -1 : nres;
        if (err) atomicOr(status, err);
    }
}

// ---------------------------------------------------------------------------
// dosages.  One warp per (target haplotype, tile of 64 sites of the window).
// Lane j handles sites base+j and base+32+j.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) dosage_kernel(
    const int4 *__restrict__ matches, int cap, const int *__restrict__ nmatch,
    const int32_t *__restrict__ absperm, int K, const uint64_t *__restrict__ hapmajor_full, int wMref,
    const int32_t *__restrict__ segm, const uint8_t *__restrict__ common, const float *__restrict__ af,
    int nrefhaps_total, const uint64_t *__restrict__ phased, int wM, const uint8_t *__restrict__ gt, int M,
    int nhaps, int mref_begin, int nsites, int imputeCalls, float *__restrict__ dos, int ldd,
    uint64_t *__restrict__ bits, int ldb) {
    const int lane = threadIdx.x & 31;
    const long gw = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int ntiles = (nsites + 63) / 64;
    const int hap = (int)(gw / ntiles);
    const int tile = (int)(gw % ntiles);
    if (hap >= nhaps) return;
    const int base = mref_begin + tile * 64;
    const int end = mref_begin + nsites;
    const uint8_t *g = gt + (size_t)(hap >> 1) * M;
    const uint64_t *hw = phased + (size_t)hap * wM;

    int s[2] = {base + lane, base + 32 + lane};
    bool valid[2], imp[2];
    int k[2];
    float afv[2];
    bool shortc[2];
    uint64_t score[2] = {0, 0}, sum[2] = {0, 0};
    for (int j = 0; j < 2; j++) {
        valid[j] = s[j] < end;
        int ss = valid[j] ? s[j] : base;
        k[j] = segm[ss];
        afv[j] = af[ss];
        imp[j] = valid[j] && (!common[ss] || g[k[j]] == 3 || imputeCalls);
    }
    // matches covering any site of the tile
    const int n = nmatch[hap] < 0 ? 0 : nmatch[hap];
    const int4 *mt = matches + (size_t)hap * cap;
    const int kmin = segm[base];
    const int kmax = segm[min(base + 63, end - 1)];
    int lo = 0, hi = n;
    {   // first match with end > kmin
        int a = 0, b = n;
        while (a < b) { int c = (a + b) >> 1; if (mt[c].y > kmin) b = c; else a = c + 1; }
        lo = a;
        a = lo; b = n;   // first match with start > kmax
        while (a < b) { int c = (a + b) >> 1; if (mt[c].x > kmax) b = c; else a = c + 1; }
        hi = a;
    }
    const int w0 = base >> 6;
    for (int i = lo; i < hi; i++) {
        const int4 mm = mt[i];
        const int height = mm.w - mm.z + 1;
        bool cov[2];
        bool loop = false;
        uint64_t single[2];
        for (int j = 0; j < 2; j++) {
            cov[j] = imp[j] && mm.x <= k[j] && k[j] < mm.y;
            single[j] = (uint64_t)(k[j] - mm.x + 1) * (uint64_t)(mm.y - k[j]);
            float maf = afv[j] > 0.5f ? 1.0f - afv[j] : afv[j];
            // TargetImp.cpp:526: float maf * Nrefhaps (as float) against double 0.01 * height
            shortc[j] = (double)__fmul_rn(maf, (float)nrefhaps_total) < 0.01 * (double)height;
            if (cov[j] && shortc[j]) {
                sum[j] += (uint64_t)height * single[j];
                if (afv[j] > 0.5f) score[j] += (uint64_t)height * single[j];
            }
            loop |= cov[j] && !shortc[j];
        }
        if (!__any_sync(0xffffffffu, loop)) continue;
        const int32_t *ap = absperm + (size_t)mm.y * K;
        for (int r = mm.z; r <= mm.w; r++) {
            const int ref = ap[r];
            const uint64_t *hr = hapmajor_full + (size_t)ref * wMref;
            const uint64_t wa = hr[w0];
            const uint64_t wb = (w0 + 1 < wMref) ? hr[w0 + 1] : 0ull;
            for (int j = 0; j < 2; j++) {
                if (cov[j] && !shortc[j]) {
                    int off = s[j] - (w0 << 6);
                    uint64_t word = off < 64 ? wa : wb;
                    sum[j] += single[j];
                    if ((word >> (off & 63)) & 1ull) score[j] += single[j];
                }
            }
        }
    }
    float* drow = dos + (size_t)hap * ldd;
    uint32_t bw[2];
    for (int j = 0; j < 2; j++) {
        int b = 0;
        float d = 0.0f;
        if (valid[j]) {
            if (imp[j]) {
                if (sum[j] == 0) d = -1.0f;           // DOSAGE_CONFLICT (TargetImp.cpp:26,507-509)
                else {
                    b = score[j] > sum[j] / 2;
                    d = (float)((double)score[j] / (double)sum[j]);
                }
            } else {
                b = bit_at(hw, k[j]);
                d = b ? 1.0f : 0.0f;
            }
            drow[s[j] - mref_begin] = d;
        }
        bw[j] = __ballot_sync(0xffffffffu, b);
    }
    if (lane == 0) bits[(size_t)hap * ldb + tile] = (uint64_t)bw[0] | ((uint64_t)bw[1] << 32);
}

// per-site segment map: segm[mref] = index of the last typed site <= mref
// (0 before the first), common[mref] = 1 at typed sites
__global__ void segmap_kernel(const int64_t *__restrict__ typed, int M, int Mref, int32_t *__restrict__ segm,
                              uint8_t *__restrict__ common) {
    int mref = blockIdx.x * blockDim.x + threadIdx.x;
    if (mref >= Mref) return;
    int a = 0, b = M;   // number of typed sites <= mref
    while (a < b) { int c = (a + b) >> 1; if (typed[c] <= mref) a = c + 1; else b = c; }
    int cnt = a;
    segm[mref] = cnt > 0 ? cnt - 1 : 0;
    common[mref] = (cnt > 0 && typed[cnt - 1] == mref) ? 1 : 0;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
size_t refpbwt_smem(int K, int wN) {
    int nwords = (K + 31) / 32;
    return (size_t)2 * wN * 4 + (size_t)nwords * 4 + (size_t)(nwords + 1) * 4 + 33 * 4;
}

cudaError_t launch_refpbwt(const uint64_t *sitemajor, int M, int K, int wN, uint32_t *compr, int32_t *absperm,
                           int32_t *count0, cudaStream_t st) {
    size_t sm = refpbwt_smem(K, wN);
    cudaError_t e = cudaFuncSetAttribute(refpbwt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    refpbwt_kernel<<<1, 1024, sm, st>>>(sitemajor, M, K, wN, compr, absperm, count0);
    return cudaGetLastError();
}

cudaError_t launch_transpose(const uint64_t *src, size_t rows, size_t srcw, uint64_t *dst, size_t cols, size_t dstw,
                             cudaStream_t st) {
    dim3 grid((unsigned)((rows + 63) / 64), (unsigned)srcw);
    transpose_kernel<<<grid, 64, 0, st>>>(src, rows, srcw, dst, cols, dstw);
    return cudaGetLastError();
}

cudaError_t launch_smm(const uint32_t *compr, const int32_t *count0, int M, int K, const uint64_t *phased, int wM,
                       const uint8_t *gt, int nhaps, int setmaxerrors, int4 *matches, int cap, int *nmatch,
                       uint32_t *status, cudaStream_t st) {
    size_t sm = sizeof(SmmWarpSmem) * SMM_WARPS;
    cudaError_t e = cudaFuncSetAttribute(smm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    int blocks = (nhaps + SMM_WARPS - 1) / SMM_WARPS;
    smm_kernel<<<blocks, SMM_WARPS * 32, sm, st>>>(compr, count0, M, K, phased, wM, gt, nhaps, setmaxerrors,
                                                   matches, cap, nmatch, status);
    return cudaGetLastError();
}

cudaError_t launch_dosage(const int4 *matches, int cap, const int *nmatch, const int32_t *absperm, int K,
                          const uint64_t *hapmajor_full, int wMref, const int32_t *segm, const uint8_t *common,
                          const float *af, int nrefhaps_total, const uint64_t *phased, int wM, const uint8_t *gt,
                          int M, int nhaps, int mref_begin, int nsites, int imputeCalls, float *dos, int ldd,
                          uint64_t *bits, int ldb, cudaStream_t st) {
    long warps = (long)nhaps * ((nsites + 63) / 64);
    long blocks = (warps + 7) / 8;
    dosage_kernel<<<(unsigned)blocks, 256, 0, st>>>(matches, cap, nmatch, absperm, K, hapmajor_full, wMref, segm,
                                                    common, af, nrefhaps_total, phased, wM, gt, M, nhaps,
                                                    mref_begin, nsites, imputeCalls, dos, ldd, bits, ldb);
    return cudaGetLastError();
}

cudaError_t launch_segmap(const int64_t *typed, int M, int Mref, int32_t *segm, uint8_t *common, cudaStream_t st) {
    segmap_kernel<<<(Mref + 255) / 256, 256, 0, st>>>(typed, M, Mref, segm, common);
    return cudaGetLastError();
}

}  // namespace eimp
