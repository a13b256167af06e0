// PBWT imputation kernels for B200 (sm_100a).
//
//  refpbwt_kernel   -- PBWT::buildComprPBWT with refPBWT=true (PBWT.cpp:207-285,
//                      136-142): compressed rows + prefix arrays gAbsPerm.
//  transpose_kernel -- site-major -> haplotype-major bit matrix (64x64 tiles).
//  smm_kernel,      -- TargetImp::calcSMMatches / processHistorySubTree
//  smm_compact_kernel  (TargetImp.cpp:74-246, 346-435), one warp per target
//                      haplotype: the rank queries of all tree nodes of a
//                      site and the rebuild of the tree run across the lanes;
//                      the compact kernel stores the tree in 30 B per node
//                      (typed sites < 65536).
//  dosage_kernel    -- TargetImp::imputeBunch (TargetImp.cpp:474-558), one
//                      warp per (target haplotype, span of 64-site tiles).
#include <climits>

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
// reference PBWT with prefix arrays, in two passes.
//
// The order before site m+1 is the order before site m, stably partitioned by
// the haplotypes' bits at site m; so the order before site m+n is the order
// before m stably sorted by the n-bit key (b[m+n-1] ... b[m+1] b[m]), the
// last site most significant.  The checkpoint pass (one CTA) walks the sites
// RP_BITS at a time with that 32-bucket stable sort and stores only the order
// before every RP_CK-th site; the fill pass (one CTA per RP_CK sites) starts
// from its checkpoint and steps site by site, writing every prefix array,
// compressed row and zero count of its interval.
// ---------------------------------------------------------------------------
constexpr int RP_CK = 64;     // sites between checkpoint orders
constexpr int RP_BITS = 5;    // sites per step of the checkpoint pass: 32 buckets, one per lane
// rounds of 32 positions whose loads are issued together: 8 with the orders
// in global memory (their latency overlapped), 1 in shared memory (fewer
// registers and instructions measured faster there)

// The orders (cur, nxt) and the step's keys live in shared memory, or in
// global scratch (2K int32 + K bytes) when 'scratch' is given; the step's
// site rows are staged in shared memory when 'stage_rows' is set.
template <int RP_U>
__global__ void __launch_bounds__(1024, 1) refpbwt_ckpt_kernel(const uint64_t *__restrict__ sitemajor, int M, int K,
                                                               int wN, int32_t *__restrict__ absperm,
                                                               int32_t *scratch, int stage_rows) {
    extern __shared__ uint64_t rp_smem[];
    int *hist = reinterpret_cast<int *>(rp_smem);   // [bucket][warp], 32 x 32
    int *wsum = hist + 1024;                        // 32
    uint64_t *rows = rp_smem + (1024 + 32) / 2;     // RP_BITS * wN when staged
    char *tail = reinterpret_cast<char *>(rows + (stage_rows ? (size_t)RP_BITS * wN : 0));
    int32_t *cur, *nxt;
    uint8_t *keys;
    if (scratch) {
        cur = scratch; nxt = scratch + K; keys = reinterpret_cast<uint8_t *>(scratch + 2 * (size_t)K);
    } else {
        cur = reinterpret_cast<int32_t *>(tail); nxt = cur + K; keys = reinterpret_cast<uint8_t *>(nxt + K);
    }
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int per = ((K + 1023) / 1024) * 32;   // elements per warp, a multiple of 32
    const int lo = min(K, w * per), hi = min(K, lo + per);
    if (M <= 0) {
        for (int i = tid; i < K; i += 1024) absperm[i] = i;
        return;
    }
    for (int i = tid; i < K; i += 1024) cur[i] = i;
    __syncthreads();
    for (int m = 0; m < M;) {
        const int nb = min(RP_BITS, min(M - m, RP_CK - m % RP_CK));
        if (m % RP_CK == 0) {
            int32_t *out = absperm + (size_t)m * K;
            for (int i = tid; i < K; i += 1024) out[i] = cur[i];
        }
        const uint64_t *rw = sitemajor + (size_t)m * wN;   // rows m .. m+nb-1 are contiguous
        if (stage_rows) {
            for (int i = tid; i < nb * wN; i += 1024) rows[i] = rw[i];
            rw = rows;
            __syncthreads();
        }
        // pass 1: keys and the per-warp bucket counts (lane b counts bucket b);
        // the orders of RP_U rounds are loaded before any is used, so that
        // their latencies overlap when the orders are in global memory
        int cnt = 0;
        for (int i00 = lo; i00 < hi; i00 += 32 * RP_U) {
            int hv[RP_U];
#pragma unroll
            for (int u = 0; u < RP_U; u++) {
                const int i = i00 + u * 32 + lane;
                hv[u] = i < hi ? cur[i] : 0;
            }
#pragma unroll
            for (int u = 0; u < RP_U; u++) {
                const int i = i00 + u * 32 + lane;
                const bool ok = i < hi;
                int key = 0;
                if (ok) {
                    const int h = hv[u];
                    for (int j = 0; j < nb; j++) key |= (int)((rw[(size_t)j * wN + (h >> 6)] >> (h & 63)) & 1) << j;
                    keys[i] = (uint8_t)key;
                }
                unsigned mine = __ballot_sync(0xffffffffu, ok);
#pragma unroll
                for (int j = 0; j < RP_BITS; j++) {
                    const unsigned bj = __ballot_sync(0xffffffffu, (key >> j) & 1);
                    mine &= ((lane >> j) & 1) ? bj : ~bj;
                }
                cnt += __popc(mine);
            }
        }
        hist[lane * 32 + w] = cnt;
        __syncthreads();
        // exclusive scan, bucket-major: the next order holds bucket 0 of
        // every warp (in warp order) first, then bucket 1, ...
        {
            const int v = hist[tid];
            int x = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) wsum[w] = x;
            __syncthreads();
            if (w == 0) {
                int z = wsum[lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, z, o);
                    if (lane >= o) z += y;
                }
                wsum[lane] = z;
            }
            __syncthreads();
            hist[tid] = x - v + (w ? wsum[w - 1] : 0);
            __syncthreads();
        }
        // pass 2: stable scatter in round order; hist[b][w] is warp w's next
        // slot of bucket b
        for (int i00 = lo; i00 < hi; i00 += 32 * RP_U) {
            int kv[RP_U], hv[RP_U];
#pragma unroll
            for (int u = 0; u < RP_U; u++) {
                const int i = i00 + u * 32 + lane;
                const bool ok = i < hi;
                kv[u] = ok ? (int)keys[i] : 32 + lane;   // past the end: a bucket of its own
                hv[u] = ok ? cur[i] : 0;
            }
#pragma unroll
            for (int u = 0; u < RP_U; u++) {
                const bool ok = i00 + u * 32 + lane < hi;
                const int key = kv[u];
                const unsigned same = __match_any_sync(0xffffffffu, key);
                const int rank = __popc(same & ((1u << lane) - 1u));
                int base = 0;
                if (ok) {
                    base = hist[key * 32 + w];
                    nxt[base + rank] = hv[u];
                }
                __syncwarp();
                if (ok && rank == 0) hist[key * 32 + w] = base + __popc(same);
                __syncwarp();
            }
        }
        __syncthreads();
        int32_t *t = cur; cur = nxt; nxt = t;
        m += nb;
    }
}

// Fill pass: CTA c covers sites [c*RP_CK, min(M, (c+1)*RP_CK)); the order
// before its first site is the checkpoint.  Per site: the bits in prefix
// order (one ballot per 32 positions), the zeros per 32-position word and
// their exclusive scan give the compressed row [data, cumulative zeros] and
// the stable partition into the next order (PBWT.cpp:207-285).
__global__ void __launch_bounds__(1024) refpbwt_fill_kernel(const uint64_t *__restrict__ sitemajor, int M, int K,
                                                           int wN, uint32_t *__restrict__ compr,
                                                           int32_t *__restrict__ absperm,
                                                           int32_t *__restrict__ count0) {
    extern __shared__ uint8_t smem[];
    const int nwords = (K + 31) / 32;
    uint32_t *row = reinterpret_cast<uint32_t *>(smem);                  // 2*wN u32
    uint32_t *data = row + 2 * wN;                                       // nwords
    int *pz = reinterpret_cast<int *>(data + nwords);                    // nwords + 1
    int *warpbuf = pz + nwords + 1;                                      // 32
    int *tot = warpbuf + 32;                                             // 1
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
    const size_t kw = 2 * (size_t)nwords;
    const int m0 = blockIdx.x * RP_CK, m1 = min(M, m0 + RP_CK);

    for (int m = m0; m < m1; m++) {
        const uint64_t *src = sitemajor + (size_t)m * wN;
        for (int w = tid; w < wN; w += blockDim.x) {
            uint64_t x = src[w];
            row[2 * w] = (uint32_t)x;
            row[2 * w + 1] = (uint32_t)(x >> 32);
        }
        __syncthreads();
        const int32_t *perm = absperm + (size_t)m * K;
        int32_t *nperm = absperm + (size_t)(m + 1) * K;
        // the order before the next checkpoint site exists already
        const bool put = !((m + 1) % RP_CK == 0 && m + 1 < M);
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
            if (i < K && put) {
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
// bit-matrix transpose: src (rows of src_ld words, 'cols' valid bits per row)
// -> dst (cols rows of dst_ld words, of which the first dstw are written:
// word w of dst row c holds bit c of src rows 64w .. 64w+63).  One 64x64 tile
// per block of 64 threads; grid (ceil(rows/64), ceil(cols/64)).
// ---------------------------------------------------------------------------
__global__ void transpose_kernel(const uint64_t *__restrict__ src, size_t rows, size_t src_ld,
                                 uint64_t *__restrict__ dst, size_t cols, size_t dstw, size_t dst_ld) {
    __shared__ uint64_t tile[64];
    const size_t rw = blockIdx.x;      // 64-row block (source rows -> dest word)
    const size_t cw = blockIdx.y;      // source word (-> 64 dest rows)
    const int t = threadIdx.x;
    size_t r = rw * 64 + t;
    tile[t] = r < rows ? src[r * src_ld + cw] : 0ull;
    __syncthreads();
    size_t c = cw * 64 + t;
    if (c < cols && rw < dstw) {
        uint64_t o = 0;
#pragma unroll 8
        for (int j = 0; j < 64; j++) o |= ((tile[j] >> t) & 1ull) << j;
        dst[c * dst_ld + rw] = o;
    }
}

// ---------------------------------------------------------------------------
// set-maximal matches
//
// TargetImp::calcSMMatches / processHistorySubTree (TargetImp.cpp:74-246,
// 346-435) keep a tree of PBWT intervals.  Two facts make the per-site update
// of that tree data-parallel:
//  * a node's descendants hold sub-intervals of its interval and at least its
//    number of errors, so a descendant can extend only if the node can;
//  * the 1-extensions are built as a mirror of the tree (TargetImp.cpp:370-388).
// Hence, with the tree stored in pre-order, one site turns the pre-order array
// O into  [new root] ++ {v in O : v extends with 0} ++ {v in O : v extends
// with 1}  (mapped intervals, depth + 1), each part keeping the relative order,
// sides and parents of O; nodes that extend neither way are deleted and, when
// at the maximum depth, report matches in pre-order; a node with exactly one
// child of equal interval and errors is replaced by that child, which in
// pre-order is the next entry.  One warp handles one target haplotype; the
// filters, scans and parent remaps run across the lanes.
// ---------------------------------------------------------------------------
struct SNode {
    int l, r;
    int de;                 // depth | errors << 24
    short parent;           // index in the array, -1 for the root
    unsigned char side;     // 0: left child, 1: right child of the parent
    unsigned char pad;
};

template <int NODES> struct SmmWarpSmem {
    SNode A[NODES];         // tree in pre-order
    SNode B[NODES];         // tree being built
    int4 mp[NODES];         // mappings (to0, to1); reused by the merge pass
    short idx0[NODES];      // position of a node's 0-extension in B (-1: none)
    short idx1[NODES];      // position of a node's 1-extension in B (-1: none)
};

__device__ __forceinline__ int de_depth(int de) { return de & 0xffffff; }
__device__ __forceinline__ int de_err(int de) { return (int)((unsigned)de >> 24); }
__device__ __forceinline__ unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }

// A match search runs first with a small node pool (many warps per SM); a
// haplotype whose tree outgrows it ends with its match count set to
// SMM_RETRY and no error, and a second launch with a large pool (one warp
// per CTA) redoes exactly those haplotypes.  Only a tree that outgrows the
// large pool too is an error (EIMP_ERR_NODE_OVERFLOW).  set-maximal errors
// make the trees grow: on a 5000-haplotype panel at 2000 sites the largest
// trees held 148, 718, 1733 and 3093 nodes at 0, 1, 2 and 3 errors.
constexpr int SMM_RETRY = -2;
__device__ __forceinline__ void smm_finish(int lane, uint32_t err, bool retry_pass, int nres, int *nmatch, int hap,
                                           uint32_t *status) {
    if (lane) return;
    if (!err) { nmatch[hap] = nres; return; }
    if (!retry_pass && err == EIMP_ERR_NODE_OVERFLOW) { nmatch[hap] = SMM_RETRY; return; }
    nmatch[hap] = -1;
    atomicOr(status, err);
}

template <int NODES, int WARPS, bool RETRY>
__global__ void __launch_bounds__(WARPS * 32) smm_kernel(
    const uint32_t *__restrict__ compr, const int32_t *__restrict__ count0, int M, int K,
    const uint64_t *__restrict__ phased, int wM, const uint8_t *__restrict__ gt, int nhaps,
    const int32_t *__restrict__ hapmap, int setmaxerrors, int4 *__restrict__ matches, int cap,
    int *__restrict__ nmatch, uint32_t *__restrict__ status) {
    extern __shared__ uint8_t smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int hi = blockIdx.x * WARPS + wid;
    if (hi >= nhaps) return;
    const int hap = hapmap ? hapmap[hi] : hi;   // the haplotypes that exist (PBWTImputer.cpp:130)
    if (RETRY && nmatch[hap] != SMM_RETRY) return;
    SmmWarpSmem<NODES> &S = reinterpret_cast<SmmWarpSmem<NODES> *>(smem_raw)[wid];
    const uint8_t *g = gt + (size_t)(hap >> 1) * M;
    const uint64_t *hw = phased + (size_t)hap * wM;
    int4 *out = matches + (size_t)hap * cap;
    const size_t kw = eimp_kw(K);
    const unsigned FULL = 0xffffffffu;

    // missingness > 50 %: no matches (TargetImp.cpp:79-80)
    int nmiss = 0;
    for (int m = lane; m < M; m += 32) nmiss += g[m] == 3;
    for (int o = 16; o; o >>= 1) nmiss += __shfl_xor_sync(FULL, nmiss, o);
    if (nmiss > M / 2) { if (lane == 0) nmatch[hap] = 0; return; }

    uint32_t err = 0;
    int n = 1, nres = 0, td = 0;
    if (lane == 0) { S.A[0].l = 0; S.A[0].r = K - 1; S.A[0].de = 0; S.A[0].parent = -1; S.A[0].side = 0; }
    __syncwarp();

    for (int m = 0; m <= M; m++) {
        const bool final = (m == M);   // TargetImp.cpp:144: erase pass, every node reports
        const int curr = final ? 0 : bit_at(hw, m);
        const int missing = final ? 0 : (g[m] == 3);
        const uint32_t *crow = compr + (size_t)(final ? 0 : m) * kw;
        const int c0 = final ? 0 : count0[m];
        // pass 1: mappings, extension flags, matches of nodes that end here
        int cnt0 = 0, cnt1 = 0, newcount = 0;
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            bool e0 = false, e1 = false, dead = false;
            if (i < n) {
                const SNode v = S.A[i];
                int l0 = 0, r0 = -1, l1 = 0, r1 = -1;
                if (!final) pbwt_map(crow, c0, v.l, v.r, l0, r0, l1, r1);
                const int ne = de_err(v.de);
                e0 = l0 <= r0 && (missing || !curr || ne < setmaxerrors);
                e1 = l1 <= r1 && (missing || curr || ne < setmaxerrors);
                S.mp[i] = make_int4(l0, r0, l1, r1);
                dead = !e0 && !e1 && de_depth(v.de) == td && td > 0;
            }
            const unsigned b0 = __ballot_sync(FULL, e0), b1 = __ballot_sync(FULL, e1), bd = __ballot_sync(FULL, dead);
            if (i < n) {
                S.idx0[i] = e0 ? (short)(1 + cnt0 + __popc(b0 & lanemask_lt())) : (short)-1;
                S.idx1[i] = e1 ? (short)(cnt1 + __popc(b1 & lanemask_lt())) : (short)-1;   // offset added below
            }
            if (dead) {
                const SNode v = S.A[i];
                const int d = de_depth(v.de);
                const int pos = nres + newcount + __popc(bd & lanemask_lt());
                if (pos < cap) out[pos] = make_int4(m - d, m, v.l, v.r);
                else err |= EIMP_ERR_MATCH_OVERFLOW;
            }
            cnt0 += __popc(b0); cnt1 += __popc(b1); newcount += __popc(bd);
        }
        __syncwarp();
        if (final) {
            if (nres + newcount <= cap) nres += newcount;
            break;
        }
        const int nb = 1 + cnt0 + cnt1;
        if (nb > NODES) { err |= EIMP_ERR_NODE_OVERFLOW; break; }
        // pass 2: build B = [new root] ++ 0-tree ++ 1-tree
        for (int i = lane; i < n; i += 32) {
            const SNode v = S.A[i];
            const int4 mp = S.mp[i];
            const int d = de_depth(v.de) + 1, ne = de_err(v.de);
            const int p0 = S.idx0[i], p1 = S.idx1[i];
            if (p0 >= 0) {
                SNode &o = S.B[p0];
                o.l = mp.x; o.r = mp.y;
                o.de = d | (((curr && !missing) ? ne + 1 : ne) << 24);
                o.parent = i == 0 ? 0 : S.idx0[v.parent];
                o.side = i == 0 ? 0 : v.side;
            }
            if (p1 >= 0) {
                SNode &o = S.B[1 + cnt0 + p1];
                o.l = mp.z; o.r = mp.w;
                o.de = d | (((!curr && !missing) ? ne + 1 : ne) << 24);
                o.parent = i == 0 ? 0 : (short)(1 + cnt0 + S.idx1[v.parent]);
                o.side = i == 0 ? 1 : v.side;
            }
        }
        if (lane == 0) { S.B[0].l = 0; S.B[0].r = K - 1; S.B[0].de = 0; S.B[0].parent = -1; S.B[0].side = 0; }
        __syncwarp();
        // pass 3: merges (TargetImp.cpp:405-432).  Child flags first.
        int *cflag = reinterpret_cast<int *>(S.mp);   // mp[i].x
        for (int i = lane; i < nb; i += 32) S.mp[i].x = 0;
        __syncwarp();
        for (int u = 1 + lane; u < nb; u += 32) atomicOr(&S.mp[S.B[u].parent].x, 1 << S.B[u].side);
        __syncwarp();
        (void)cflag;
        // removal flags, kept-position scan, start of each removed run
        int kept = 0, laststart = -1;
        for (int base = 0; base < nb; base += 32) {
            const int v = base + lane;
            bool rm = false, start = false;
            if (v >= 1 && v < nb) {
                const int cf = S.mp[v].x;
                if (cf == 1 || cf == 2) {   // exactly one child: the next entry
                    const SNode a = S.B[v], c = S.B[v + 1];
                    rm = a.l == c.l && a.r == c.r && de_err(a.de) == de_err(c.de);
                }
            }
            const unsigned brm = __ballot_sync(FULL, rm);
            // a removed run starts where the previous entry is kept
            const unsigned prevrm = (brm << 1) | (base > 0 ? (unsigned)((S.mp[base - 1].w >> 1) & 1) : 0u);
            start = rm && !((prevrm >> lane) & 1);
            const unsigned bst = __ballot_sync(FULL, start);
            // last run start at or before this entry (inclusive prefix max)
            const unsigned upto = bst & (lanemask_lt() | (1u << lane));
            const int ls = upto ? base + (31 - __clz(upto)) : laststart;
            const bool keep = v < nb && !rm;
            const unsigned bk = __ballot_sync(FULL, keep);
            if (v < nb) S.mp[v] = make_int4(S.mp[v].x, keep ? kept + __popc(bk & lanemask_lt()) : -1, ls,
                                            rm ? 2 : 0);
            kept += __popc(bk);
            if (bst) laststart = base + (31 - __clz(bst));
            __syncwarp();
        }
        // compact into A with remapped parents
        for (int u = lane; u < nb; u += 32) {
            const int np = S.mp[u].y;
            if (np < 0) continue;
            SNode o = S.B[u];
            if (u > 0) {
                int p = o.parent;
                if (S.mp[p].w & 2) {   // parent removed: take the place of its run's first node
                    const int q = S.mp[p].z;
                    p = S.B[q].parent;
                    o.side = S.B[q].side;
                }
                o.parent = (short)S.mp[p].y;
            }
            S.A[np] = o;
        }
        __syncwarp();
        n = kept;
        int md = 0;
        for (int i = lane; i < n; i += 32) md = max(md, de_depth(S.A[i].de));
        for (int o = 16; o; o >>= 1) md = max(md, __shfl_xor_sync(FULL, md, o));
        // TargetImp.cpp:132-136: the site's matches are set-maximal only if no
        // longer path is still alive
        if (newcount && td >= md && nres + newcount <= cap) nres += newcount;
        td = md;
    }
    for (int o = 16; o; o >>= 1) err |= __shfl_xor_sync(FULL, err, o);
    smm_finish(lane, err, RETRY, nres, nmatch, hap, status);
}

// ---------------------------------------------------------------------------
// The same set-maximal match search with a compact tree (typed sites < 65536):
// structure of arrays with the depth in 16 bits, packed with the parent index
// and side, and the errors in a byte -- 30 bytes per node instead of 52, so
// that a warp holds 15.5 KB of shared memory and 2000 target haplotypes fit
// on the device at once (14 warps per SM instead of 8).  The mapped intervals
// are not kept in an array of their own: pass 1 writes a node's 0-extension
// interval straight into the new tree and its 1-extension interval over the
// node's own interval, which pass 2 reads back; the merge pass keeps its
// bookkeeping in the extension-index arrays.  Same algorithm and output as
// smm_kernel above.
// ---------------------------------------------------------------------------
// IV: the interval bounds' type -- 16 bits when the reference PBWT holds at
// most 65,536 haplotypes (22 bytes per node instead of 30, so more warps fit
// an SM), else 32 bits.  An empty extension interval stored over a node's own
// (r = -1) is never read back, so its wrap in 16 bits does no harm.
template <int NODES, typename IV> struct SmmTree {
    IV l[NODES], r[NODES];
    unsigned dps[NODES];              // depth | (parent + 1) << 16 | side << 31
    unsigned char e[NODES];           // errors
};
template <int NODES, typename IV = int> struct SmmWarpSmemC {
    SmmTree<NODES, IV> A, B;
    short idx0[NODES];                // extension positions; kept positions in the merge pass
    short idx1[NODES];                // extension positions; run starts in the merge pass
    unsigned cflag[NODES / 16];       // 2 bits per node: which children it has
};

__device__ __forceinline__ int dps_depth(unsigned x) { return (int)(x & 0xffffu); }
__device__ __forceinline__ int dps_parent(unsigned x) { return (int)((x >> 16) & 0x7fffu) - 1; }
__device__ __forceinline__ int dps_side(unsigned x) { return (int)(x >> 31); }
__device__ __forceinline__ unsigned dps_make(int depth, int parent, int side) {
    return (unsigned)depth | ((unsigned)(parent + 1) << 16) | ((unsigned)side << 31);
}

// The sites [m0, M] of one haplotype's match search on a tree pool of NODES
// nodes (S, in shared or in global memory); A is the tree, B the one being
// built.  Returns M + 1 when the haplotype is done (or its tree outgrew the
// pool: err), or -- with can_switch -- the first site whose pass could
// outgrow the pool, before touching the tree, so that the caller can move it
// to a larger pool and go on from that site.
template <int NODES, typename IV>
__device__ int smm_compact_sites(SmmWarpSmemC<NODES, IV> &S, SmmTree<NODES, IV> *&A, SmmTree<NODES, IV> *&B,
                                 int m0, bool can_switch, const uint32_t *__restrict__ compr,
                                 const int32_t *__restrict__ count0, int M, int K, size_t kw, const uint8_t *g,
                                 const uint64_t *hw, int setmaxerrors, int4 *out, int cap, int &n, int &nres, int &td,
                                 uint32_t &err) {
    const int lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    for (int m = m0; m <= M; m++) {
        const bool final = (m == M);   // TargetImp.cpp:144: erase pass, every node reports
        // a site can at most double the tree (plus the new root): hand over to
        // the larger pool before the pass that could outgrow this one
        if (can_switch && !final && 2 * n + 1 > NODES) return m;
        const int curr = final ? 0 : bit_at(hw, m);
        const int missing = final ? 0 : (g[m] == 3);
        const uint32_t *crow = compr + (size_t)(final ? 0 : m) * kw;
        const int c0 = final ? 0 : count0[m];
        // pass 1: mappings, extension flags, matches of nodes that end here;
        // the 0-extension interval goes to its place in B, the 1-extension
        // interval over the node's own
        int cnt0 = 0, cnt1 = 0, newcount = 0;
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            bool e0 = false, e1 = false, dead = false;
            int l0 = 0, r0 = -1, l1 = 0, r1 = -1, vl = 0, vr = -1, d = 0;
            if (i < n) {
                vl = A->l[i]; vr = A->r[i];
                d = dps_depth(A->dps[i]);
                const int ne = A->e[i];
                if (!final) pbwt_map(crow, c0, vl, vr, l0, r0, l1, r1);
                e0 = l0 <= r0 && (missing || !curr || ne < setmaxerrors);
                e1 = l1 <= r1 && (missing || curr || ne < setmaxerrors);
                dead = !e0 && !e1 && d == td && td > 0;
            }
            const unsigned b0 = __ballot_sync(FULL, e0), b1 = __ballot_sync(FULL, e1), bd = __ballot_sync(FULL, dead);
            if (i < n) {
                const int p0 = e0 ? 1 + cnt0 + __popc(b0 & lanemask_lt()) : -1;
                S.idx0[i] = (short)p0;
                S.idx1[i] = e1 ? (short)(cnt1 + __popc(b1 & lanemask_lt())) : (short)-1;   // offset added below
                if (p0 >= 0 && p0 < NODES) { B->l[p0] = (IV)l0; B->r[p0] = (IV)r0; }
                A->l[i] = (IV)l1; A->r[i] = (IV)r1;
            }
            if (dead) {
                const int pos = nres + newcount + __popc(bd & lanemask_lt());
                if (pos < cap) out[pos] = make_int4(m - d, m, vl, vr);
                else err |= EIMP_ERR_MATCH_OVERFLOW;
            }
            cnt0 += __popc(b0); cnt1 += __popc(b1); newcount += __popc(bd);
        }
        __syncwarp();
        if (final) {
            if (nres + newcount <= cap) nres += newcount;
            return M + 1;
        }
        const int nb = 1 + cnt0 + cnt1;
        if (nb > NODES) { err |= EIMP_ERR_NODE_OVERFLOW; return M + 1; }
        // pass 2: the rest of B = [new root] ++ 0-tree ++ 1-tree.  The largest
        // depth of B is the largest after the merges too: a merged node has a
        // child, which is deeper
        int md = 0;
        for (int i = lane; i < n; i += 32) {
            const unsigned vd = A->dps[i];
            const int d = dps_depth(vd) + 1, ne = A->e[i];
            if (S.idx0[i] >= 0 || S.idx1[i] >= 0) md = max(md, d);
            const int vp = dps_parent(vd), vs = dps_side(vd);
            const int p0 = S.idx0[i], p1 = S.idx1[i];
            if (p0 >= 0) {
                B->dps[p0] = dps_make(d, i == 0 ? 0 : S.idx0[vp], i == 0 ? 0 : vs);
                B->e[p0] = (unsigned char)((curr && !missing) ? ne + 1 : ne);
            }
            if (p1 >= 0) {
                const int q = 1 + cnt0 + p1;
                B->l[q] = A->l[i]; B->r[q] = A->r[i];
                B->dps[q] = dps_make(d, i == 0 ? 0 : 1 + cnt0 + S.idx1[vp], i == 0 ? 1 : vs);
                B->e[q] = (unsigned char)((!curr && !missing) ? ne + 1 : ne);
            }
        }
        if (lane == 0) { B->l[0] = 0; B->r[0] = (IV)(K - 1); B->dps[0] = dps_make(0, -1, 0); B->e[0] = 0; }
        for (int q = lane; q < (nb + 15) / 16; q += 32) S.cflag[q] = 0u;
        __syncwarp();
        // pass 3: merges (TargetImp.cpp:405-432).  Child flags first.
        for (int u = 1 + lane; u < nb; u += 32) {
            const unsigned x = B->dps[u];
            const int pa = dps_parent(x);
            atomicOr(&S.cflag[pa >> 4], (1u << dps_side(x)) << ((pa & 15) * 2));
        }
        __syncwarp();
        // removal flags, kept-position scan (-> idx0, -1 when removed), start
        // of each removed run (-> idx1)
        int kept = 0, laststart = -1;
        for (int base = 0; base < nb; base += 32) {
            const int v = base + lane;
            bool rm = false;
            if (v >= 1 && v < nb) {
                const unsigned cf = (S.cflag[v >> 4] >> ((v & 15) * 2)) & 3u;
                if (cf == 1u || cf == 2u)   // exactly one child: the next entry
                    rm = B->l[v] == B->l[v + 1] && B->r[v] == B->r[v + 1] && B->e[v] == B->e[v + 1];
            }
            const unsigned brm = __ballot_sync(FULL, rm);
            // a removed run starts where the previous entry is kept
            const unsigned prevrm = (brm << 1) | (base > 0 ? (unsigned)(S.idx0[base - 1] < 0) : 0u);
            const bool start = rm && !((prevrm >> lane) & 1u);
            const unsigned bst = __ballot_sync(FULL, start);
            const unsigned upto = bst & (lanemask_lt() | (1u << lane));
            const int ls = upto ? base + (31 - __clz(upto)) : laststart;
            const bool keep = v < nb && !rm;
            const unsigned bk = __ballot_sync(FULL, keep);
            __syncwarp();   // every lane has read idx0[base - 1]
            if (v < nb) {
                S.idx0[v] = keep ? (short)(kept + __popc(bk & lanemask_lt())) : (short)-1;
                S.idx1[v] = (short)ls;
            }
            kept += __popc(bk);
            if (bst) laststart = base + (31 - __clz(bst));
            __syncwarp();
        }
        // compact into A with remapped parents, or take B as it is
        for (int u = lane; kept < nb && u < nb; u += 32) {
            const int np = S.idx0[u];
            if (np < 0) continue;
            unsigned x = B->dps[u];
            if (u > 0) {
                int p = dps_parent(x), side = dps_side(x);
                if (S.idx0[p] < 0) {   // parent removed: take the place of its run's first node
                    const int q = S.idx1[p];
                    const unsigned xq = B->dps[q];
                    p = dps_parent(xq);
                    side = dps_side(xq);
                }
                x = dps_make(dps_depth(x), S.idx0[p], side);
            }
            A->l[np] = B->l[u]; A->r[np] = B->r[u]; A->dps[np] = x; A->e[np] = B->e[u];
        }
        if (kept == nb) { SmmTree<NODES, IV> *t = A; A = B; B = t; }
        __syncwarp();
        n = kept;
        for (int o = 16; o; o >>= 1) md = max(md, __shfl_xor_sync(FULL, md, o));
        // TargetImp.cpp:132-136: the site's matches are set-maximal only if no
        // longer path is still alive
        if (newcount && td >= md && nres + newcount <= cap) nres += newcount;
        td = md;
    }
    return M + 1;
}

// The first launch gives each warp a shared-memory pool of NODES nodes.  A
// tree that could outgrow it moves, between two sites, to a pool of
// SMM_NODES_RETRY nodes in global memory (gpool, one slot per such warp, as
// many as gpool_slots) and the warp goes on from that site; only when no slot
// is left does the haplotype end with the retry mark for the retry launch
// (RETRY: shared pools of SMM_NODES_RETRY nodes, one warp per CTA), which
// redoes it from its first site.
template <int NODES, int WARPS, bool RETRY, typename IV>
__global__ void __launch_bounds__(WARPS * 32) smm_compact_kernel(
    const uint32_t *__restrict__ compr, const int32_t *__restrict__ count0, int M, int K,
    const uint64_t *__restrict__ phased, int wM, const uint8_t *__restrict__ gt, int nhaps,
    const int32_t *__restrict__ hapmap, int setmaxerrors, int4 *__restrict__ matches, int cap,
    int *__restrict__ nmatch, uint32_t *__restrict__ status, SmmWarpSmemC<SMM_NODES_RETRY, IV> *__restrict__ gpool,
    int gpool_slots, int *__restrict__ gpool_next) {
    extern __shared__ uint8_t smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int hi = blockIdx.x * WARPS + wid;
    if (hi >= nhaps) return;
    const int hap = hapmap ? hapmap[hi] : hi;   // the haplotypes that exist (PBWTImputer.cpp:130)
    if (RETRY && nmatch[hap] != SMM_RETRY) return;
    SmmWarpSmemC<NODES, IV> &S = reinterpret_cast<SmmWarpSmemC<NODES, IV> *>(smem_raw)[wid];
    SmmTree<NODES, IV> *A = &S.A, *B = &S.B;   // the tree and the one being built; swapped when a site merges nothing
    const uint8_t *g = gt + (size_t)(hap >> 1) * M;
    const uint64_t *hw = phased + (size_t)hap * wM;
    int4 *out = matches + (size_t)hap * cap;
    const size_t kw = eimp_kw(K);
    const unsigned FULL = 0xffffffffu;

    // missingness > 50 %: no matches (TargetImp.cpp:79-80)
    int nmiss = 0;
    for (int m = lane; m < M; m += 32) nmiss += g[m] == 3;
    for (int o = 16; o; o >>= 1) nmiss += __shfl_xor_sync(FULL, nmiss, o);
    if (nmiss > M / 2) { if (lane == 0) nmatch[hap] = 0; return; }

    uint32_t err = 0;
    int n = 1, nres = 0, td = 0;
    if (lane == 0) { A->l[0] = 0; A->r[0] = (IV)(K - 1); A->dps[0] = dps_make(0, -1, 0); A->e[0] = 0; }
    __syncwarp();
    const bool big = !RETRY && gpool != nullptr && NODES < SMM_NODES_RETRY;
    int m = smm_compact_sites<NODES, IV>(S, A, B, 0, big, compr, count0, M, K, kw, g, hw, setmaxerrors, out, cap, n,
                                         nres, td, err);
    if (m <= M) {
        int slot = 0;
        if (lane == 0) slot = atomicAdd(gpool_next, 1);
        slot = __shfl_sync(FULL, slot, 0);
        if (slot < gpool_slots) {
            // the tree (n <= NODES / 2 nodes) into the global pool, then on from site m
            SmmWarpSmemC<SMM_NODES_RETRY, IV> &G = gpool[slot];
            for (int i = lane; i < n; i += 32) {
                G.A.l[i] = A->l[i]; G.A.r[i] = A->r[i]; G.A.dps[i] = A->dps[i]; G.A.e[i] = A->e[i];
            }
            __syncwarp();
            SmmTree<SMM_NODES_RETRY, IV> *GA = &G.A, *GB = &G.B;
            smm_compact_sites<SMM_NODES_RETRY, IV>(G, GA, GB, m, false, compr, count0, M, K, kw, g, hw, setmaxerrors,
                                                  out, cap, n, nres, td, err);
        } else {
            // no slot left: on in shared memory; a tree that outgrows it is retried
            smm_compact_sites<NODES, IV>(S, A, B, m, false, compr, count0, M, K, kw, g, hw, setmaxerrors, out, cap, n,
                                         nres, td, err);
        }
    }
    for (int o = 16; o; o >>= 1) err |= __shfl_xor_sync(FULL, err, o);
    smm_finish(lane, err, RETRY, nres, nmatch, hap, status);
}

// ---------------------------------------------------------------------------
// dosages (TargetImp::imputeBunch, TargetImp.cpp:474-558).
//
// One warp per (target haplotype, span of DOS_SPAN tiles of 64 sites); lane j
// owns sites base+j and base+32+j of each tile.  A site's dosage sums, over
// the set-maximal matches covering its last typed site k (start <= k < end),
// single = (k-start+1)(end-k) once per reference of the match's interval, and
// into the score where that reference carries the alternative allele.  The
// matches are sorted by end and by start, so the warp keeps a window of 32
// of them in registers (one per lane) and slides it along the span: matches
// that end at or before a tile's first segment leave at the front, and the
// covering ones are the window's prefix up to the first match that starts
// after the tile's last segment.  The (match, reference) pairs ("slots") of
// the covering matches are dealt out to the lanes; each lane keeps its
// slot's reference haplotype for as long as the covering matches stay the
// same (usually many tiles), loads that haplotype's 64 sites of the tile (one
// word of the haplotype-major panel, two where the window is not
// word-aligned), and the per-site counts come from shuffles of those words.
// More than 32 slots or covering matches take a general path that deals the
// slots out in chunks of 32 per tile.  score and sum are integers, so the
// order of the additions does not change them and the dosage (double score /
// double sum, rounded to float) is bit-exact.
//
// Per reference site the kernel reads one int2 (sinfo, built with the
// segment map): x = last typed site k | typed-site flag << 31, y = the
// smallest match height that takes the low-frequency shortcut of
// TargetImp.cpp:522-531 (float maf * Nrefhaps < 0.01 * height, evaluated
// once per site instead of once per match) | (af > 0.5) << 31.
// ---------------------------------------------------------------------------
constexpr int DOS_SPAN = 8;   // default tiles per warp (eimp_set_launch_shape: 4, 8 or 16)

// uint64 -> double without the conversion unit: exact for x < 2^52 (the bits
// of 2^52 + x as a double, minus 2^52)
__device__ __forceinline__ double dos_u64_to_f64(uint64_t x) {
    if (x < (1ull << 52)) return __longlong_as_double((long long)(0x4330000000000000ull | x)) - 4503599627370496.0;
    return (double)x;
}

// a double q in [2^-126, 1] rounded to the nearest float, ties to even (the
// rounding of a C cast), by integer operations on its bits: keep 23 of the 52
// fraction bits, add half an ulp minus one plus the kept lowest bit, and let
// a carry out of the fraction step the exponent
__device__ __forceinline__ float dos_f64_to_f32(double q) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(q);
    const unsigned e = (unsigned)(b >> 52);
    const unsigned long long m = b & ((1ull << 52) - 1);
    const unsigned long long r = m + 0x0FFFFFFFull + ((m >> 29) & 1ull);
    return __uint_as_float(((e - 1023u + 127u) << 23) + (unsigned)(r >> 29));
}

// one covered site's share of a match: the shortcut adds height x single to
// the sum (and to the score where the alternative allele is the major one),
// otherwise single per reference of the match (n of them in this chunk,
// cnt of them with the alternative allele).  With fewer than 131,071 typed
// sites single = (k-start+1)(end-k) <= ((M+1)/2)^2 fits 32 bits and every
// term is one 32 x 32 -> 64-bit multiply-add (WIDE: 64-bit single).
template <bool WIDE> struct DosSite {
    int k, hthr;
    bool imp, altmajor;
    uint64_t score, sum;
    __device__ __forceinline__ void add(int st, int en, int h, int cnt, int n, bool first) {
        if (!imp || st > k || k >= en) return;
        if (WIDE) {
            const uint64_t single = (uint64_t)(k - st + 1) * (uint64_t)(en - k);
            if (h >= hthr) {
                if (first) {
                    const uint64_t t = (uint64_t)h * single;
                    sum += t;
                    if (altmajor) score += t;
                }
            } else {
                score += single * (uint64_t)cnt;
                sum += single * (uint64_t)n;
            }
        } else {
            const uint32_t single = (uint32_t)(k - st + 1) * (uint32_t)(en - k);
            if (h >= hthr) {
                if (first) {
                    const uint64_t t = (uint64_t)(uint32_t)h * single;
                    sum += t;
                    if (altmajor) score += t;
                }
            } else {
                score += (uint64_t)single * (uint32_t)cnt;
                sum += (uint64_t)single * (uint32_t)n;
            }
        }
    }
    __device__ __forceinline__ float dosage(int &bit) const {
        if (sum == 0) return -1.0f;   // DOSAGE_CONFLICT (TargetImp.cpp:26,507-509)
        bit = score > sum / 2;
        if (score == 0) return 0.0f;
        return dos_f64_to_f32(dos_u64_to_f64(score) / dos_u64_to_f64(sum));
    }
};

__device__ __forceinline__ void dos_word(const uint64_t *__restrict__ hr, int w0, int o0, int wMref, uint32_t &lo,
                                         uint32_t &hi) {
    uint64_t x = hr[w0];
    if (o0) x = (x >> o0) | ((w0 + 1 < wMref ? hr[w0 + 1] : 0ull) << (64 - o0));
    lo = (uint32_t)x;
    hi = (uint32_t)(x >> 32);
}

// hapmap (null: identity): the target haplotype row of each of the nhaps
// haplotypes imputed (PBWTImputer.cpp:130, 202); refmap (null: identity):
// the panel haplotype of each haplotype of the reduced reference PBWT whose
// prefix arrays absperm holds (TargetImp.cpp:536, haploidsRefMap)
template <bool WIDE, int SPAN>
__global__ void __launch_bounds__(256, 4) dosage_kernel(
    const int4 *__restrict__ matches, int cap, const int *__restrict__ nmatch,
    const int32_t *__restrict__ absperm, int K, const int32_t *__restrict__ refmap,
    const uint64_t *__restrict__ hapmajor_full, int wMref, const int2 *__restrict__ sinfo,
    const uint64_t *__restrict__ phased, int wM, const uint8_t *__restrict__ gt, int M, int nhaps,
    const int32_t *__restrict__ hapmap, int mref_begin, int nsites, int imputeCalls, float *__restrict__ dos, int ldd,
    uint64_t *__restrict__ bits, int ldb) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long gw = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int ntiles = (nsites + 63) / 64;
    const int nspans = (ntiles + SPAN - 1) / SPAN;
    const int hi = (int)(gw / nspans);
    if (hi >= nhaps) return;
    const int hap = hapmap ? hapmap[hi] : hi;
    const int t0 = (int)(gw % nspans) * SPAN, t1 = min(ntiles, t0 + SPAN);
    const int end = mref_begin + nsites;
    const uint8_t *g = gt + (size_t)(hap >> 1) * M;
    const uint64_t *hw = phased + (size_t)hap * wM;
    const int n = max(nmatch[hap], 0);
    const int4 *mt = matches + (size_t)hap * cap;
    // an empty window slot: it neither covers nor leaves
    const int4 NONE = make_int4(INT_MAX, INT_MAX, 0, -1);
    const int KMASK = 0x7fffffff;

    // window start: the first match ending after the span's first segment
    // (n if none).  The list is sorted by end, so a 32-way search narrows
    // [qlo, qhi] to at most 32 candidates in a few dependent loads (a linear
    // scan from the list's start took one per 32 matches before the span).
    const int kmin0 = sinfo[mref_begin + t0 * 64].x & KMASK;
    int qlo = 0, qhi = n;   // the answer lies in [qlo, qhi]
    while (qhi - qlo > 32) {
        const int step = (qhi - qlo + 31) >> 5;   // probes qlo, qlo + step, ..., 31 of them before qhi
        const int p = qlo + lane * step;
        const unsigned f = __ballot_sync(FULL, p >= qhi || mt[p].y > kmin0);
        const int t = f ? __ffs((int)f) - 1 : 32;   // the first probe at or past the answer
        if (t == 0) { qhi = qlo; break; }
        const int nqlo = qlo + (t - 1) * step + 1;
        if (t < 32) qhi = min(qhi, qlo + t * step);
        qlo = nqlo;
    }
    int wb = qhi;
    {
        const unsigned f = __ballot_sync(FULL, qlo + lane < qhi && mt[qlo + lane].y > kmin0);
        if (f) wb = qlo + __ffs((int)f) - 1;
    }
    int4 win = wb + lane < n ? mt[wb + lane] : NONE;
    // slots of the covering set (cwb, cncov): per window lane its height and
    // first slot, per lane its slot's reference haplotype (-1: none)
    int cwb = -1, cncov = -1, hgt = 0, off = 0, total = 0, sref = -1;

    for (int tile = t0; tile < t1; tile++) {
        const int base = mref_begin + tile * 64;
        const int kmin = sinfo[base].x & KMASK;
        const int kmax = sinfo[min(base + 63, end - 1)].x & KMASK;
        // matches ending at or before kmin leave the front of the window (TargetImp.cpp:489-490)
        for (;;) {
            const unsigned d = __ballot_sync(FULL, win.y <= kmin);
            if (!(d & 1u)) break;
            const int nd = ~d ? __ffs(~d) - 1 : 32;
            wb += nd;
            win = wb + lane < n ? mt[wb + lane] : NONE;
            if (nd < 32) break;
        }
        DosSite<WIDE> S0, S1;
        const int s0 = base + lane, s1 = base + 32 + lane;
        const bool valid0 = s0 < end, valid1 = s1 < end;
        {
            const int2 i0 = sinfo[valid0 ? s0 : base], i1 = sinfo[valid1 ? s1 : base];
            S0.k = i0.x & KMASK; S0.hthr = i0.y & KMASK; S0.altmajor = i0.y < 0;
            S1.k = i1.x & KMASK; S1.hthr = i1.y & KMASK; S1.altmajor = i1.y < 0;
            S0.imp = valid0 && (i0.x >= 0 || g[S0.k] == 3 || imputeCalls);
            S1.imp = valid1 && (i1.x >= 0 || g[S1.k] == 3 || imputeCalls);
            S0.score = S0.sum = S1.score = S1.sum = 0;
        }
        const int w0 = base >> 6, o0 = base & 63;
        // covering matches: up to the first one starting after the tile (TargetImp.cpp:516)
        const unsigned cb = __ballot_sync(FULL, win.x <= kmax);
        const int ncov = ~cb ? __ffs(~cb) - 1 : 32;
        if (ncov != cncov || wb != cwb) {
            hgt = lane < ncov ? win.w - win.z + 1 : 0;
            off = hgt;
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, off, o);
                if (lane >= o) off += t;
            }
            total = __shfl_sync(FULL, off, 31);
            off -= hgt;
            int mi = 0;   // the match of this lane's slot: the last with first slot <= lane
            for (int i = 1; i < ncov; i++) mi += __shfl_sync(FULL, off, i) <= lane;
            const int my = __shfl_sync(FULL, win.y, mi), mz = __shfl_sync(FULL, win.z, mi);
            const int mo = __shfl_sync(FULL, off, mi);
            sref = lane < total ? absperm[(size_t)my * K + mz + (lane - mo)] : -1;
            if (refmap && sref >= 0) sref = refmap[sref];
            cwb = wb;
            cncov = ncov;
        }
        if (ncov < 32 && total <= 32) {
            // every slot has its lane
            uint32_t xlo = 0u, xhi = 0u;
            if (sref >= 0) dos_word(hapmajor_full + (size_t)sref * wMref, w0, o0, wMref, xlo, xhi);
            for (int i = 0; i < ncov; i++) {
                const int oi = __shfl_sync(FULL, off, i), hi = __shfl_sync(FULL, hgt, i);
                const int st = __shfl_sync(FULL, win.x, i), en = __shfl_sync(FULL, win.y, i);
                int cnt0 = 0, cnt1 = 0;
                for (int q = oi; q < oi + hi; q++) {
                    cnt0 += (__shfl_sync(FULL, xlo, q) >> lane) & 1u;
                    cnt1 += (__shfl_sync(FULL, xhi, q) >> lane) & 1u;
                }
                S0.add(st, en, hi, cnt0, hi, true);
                S1.add(st, en, hi, cnt1, hi, true);
            }
        } else {
            // general path: pages of 32 covering matches, chunks of 32 slots
            for (int pb = 0;; pb += 32) {
                const int4 pw = pb == 0 ? win : (wb + pb + lane < n ? mt[wb + pb + lane] : NONE);
                const unsigned pc = __ballot_sync(FULL, pw.x <= kmax);
                const int pn = ~pc ? __ffs(~pc) - 1 : 32;
                if (pn == 0) break;
                const int ph = lane < pn ? pw.w - pw.z + 1 : 0;
                int po = ph;
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(FULL, po, o);
                    if (lane >= o) po += t;
                }
                const int ptot = __shfl_sync(FULL, po, 31);
                po -= ph;
                for (int c = 0; c < ptot; c += 32) {
                    const int s = c + lane;
                    int mi = 0;
                    for (int i = 1; i < pn; i++) mi += __shfl_sync(FULL, po, i) <= s;
                    const int my = __shfl_sync(FULL, pw.y, mi), mz = __shfl_sync(FULL, pw.z, mi);
                    const int mo = __shfl_sync(FULL, po, mi);
                    uint32_t xlo = 0u, xhi = 0u;
                    if (s < ptot) {
                        int ref = absperm[(size_t)my * K + mz + (s - mo)];
                        if (refmap) ref = refmap[ref];
                        dos_word(hapmajor_full + (size_t)ref * wMref, w0, o0, wMref, xlo, xhi);
                    }
                    const int cend = min(ptot, c + 32);
                    for (int i = 0; i < pn; i++) {
                        const int oi = __shfl_sync(FULL, po, i), hi = __shfl_sync(FULL, ph, i);
                        const int a = max(oi, c), b = min(oi + hi, cend);
                        if (a >= b) continue;   // warp-uniform
                        int cnt0 = 0, cnt1 = 0;
                        for (int q = a; q < b; q++) {
                            cnt0 += (__shfl_sync(FULL, xlo, q - c) >> lane) & 1u;
                            cnt1 += (__shfl_sync(FULL, xhi, q - c) >> lane) & 1u;
                        }
                        const int st = __shfl_sync(FULL, pw.x, i), en = __shfl_sync(FULL, pw.y, i);
                        S0.add(st, en, hi, cnt0, b - a, a == oi);
                        S1.add(st, en, hi, cnt1, b - a, a == oi);
                    }
                }
                if (pn < 32) break;
            }
        }

        float *drow = dos + (size_t)hap * ldd;
        int b0 = 0, b1 = 0;
        if (valid0) {
            float d;
            if (S0.imp) d = S0.dosage(b0);
            else { b0 = bit_at(hw, S0.k); d = b0 ? 1.0f : 0.0f; }
            drow[s0 - mref_begin] = d;
        }
        if (valid1) {
            float d;
            if (S1.imp) d = S1.dosage(b1);
            else { b1 = bit_at(hw, S1.k); d = b1 ? 1.0f : 0.0f; }
            drow[s1 - mref_begin] = d;
        }
        const unsigned bw0 = __ballot_sync(FULL, b0), bw1 = __ballot_sync(FULL, b1);
        if (lane == 0) bits[(size_t)hap * ldb + tile] = (uint64_t)bw0 | ((uint64_t)bw1 << 32);
    }
}

// per-site segment map: segm[mref] = index of the last typed site <= mref
// (0 before the first), common[mref] = 1 at typed sites; sinfo[mref] (the
// dosage kernel's per-site word pair) = {segm | common << 31, the smallest
// match height h with (double)(float maf * (float)Nrefhaps) < 0.01 * (double)h
// -- the low-frequency shortcut of TargetImp.cpp:526 -- | (af > 0.5) << 31}
__global__ void segmap_kernel(const int64_t *__restrict__ typed, int M, int Mref, const float *__restrict__ af,
                              int nrefhaps_total, int32_t *__restrict__ segm, uint8_t *__restrict__ common,
                              int2 *__restrict__ sinfo) {
    int mref = blockIdx.x * blockDim.x + threadIdx.x;
    if (mref >= Mref) return;
    int a = 0, b = M;   // number of typed sites <= mref
    while (a < b) { int c = (a + b) >> 1; if (typed[c] <= mref) a = c + 1; else b = c; }
    int cnt = a;
    const int k = cnt > 0 ? cnt - 1 : 0;
    const int cm = (cnt > 0 && typed[cnt - 1] == mref) ? 1 : 0;
    segm[mref] = k;
    common[mref] = (uint8_t)cm;
    const float afv = af[mref];
    const float maf = afv > 0.5f ? 1.0f - afv : afv;
    const double x = (double)__fmul_rn(maf, (float)nrefhaps_total);
    // 0.01 * h is monotone in h: step up from just below x / 0.01
    double start = floor(x * 100.0) - 2.0;
    int h = start < 1.0 ? 1 : (start > 1.0e9 ? 1000000000 : (int)start);
    while (h < 1000000000 && !(x < 0.01 * (double)h)) h++;
    sinfo[mref] = make_int2(k | (cm << 31), h | ((afv > 0.5f ? 1 : 0) << 31));
}

// rows of a bit matrix gathered by index: dst[i] = src[idx[i]] (w words each)
__global__ void gather_rows_kernel(const uint64_t *__restrict__ src, size_t ldsrc, const int64_t *__restrict__ idx,
                                   int n, int w, uint64_t *__restrict__ dst) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)n * w) return;
    const int r = (int)(i / w), c = (int)(i % w);
    dst[i] = src[(size_t)idx[r] * ldsrc + c];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static size_t refpbwt_fill_smem(int K, int wN) {
    int nwords = (K + 31) / 32;
    return (size_t)2 * wN * 4 + (size_t)nwords * 4 + (size_t)(nwords + 1) * 4 + 33 * 4;
}

// shared memory of the checkpoint pass: counts and scan sums, the staged
// rows, and (without scratch) the two orders and the keys
static size_t refpbwt_ckpt_smem(int K, int wN, bool stage_rows, bool in_smem) {
    return (size_t)(1024 + 32) * 4 + (stage_rows ? (size_t)RP_BITS * wN * 8 : 0) +
           (in_smem ? (size_t)K * 9 : 0);
}

static int optin_smem() {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return 0;
    return v;
}

size_t refpbwt_scratch_bytes(int K, int wN) {
    const size_t lim = (size_t)optin_smem();
    return refpbwt_ckpt_smem(K, wN, true, true) <= lim ? 0 : (size_t)K * 9;
}

cudaError_t launch_refpbwt(const uint64_t *sitemajor, int M, int K, int wN, uint32_t *compr, int32_t *absperm,
                           int32_t *count0, int32_t *scratch, cudaStream_t st) {
    const size_t lim = (size_t)optin_smem();
    const bool in_smem = refpbwt_ckpt_smem(K, wN, true, true) <= lim;
    if (!in_smem && !scratch) return cudaErrorInvalidValue;
    const bool stage = refpbwt_ckpt_smem(K, wN, true, in_smem) <= lim;
    size_t sm = refpbwt_ckpt_smem(K, wN, stage, in_smem);
    auto ck = in_smem ? refpbwt_ckpt_kernel<1> : refpbwt_ckpt_kernel<8>;
    cudaError_t e = ensure_dynamic_smem((const void *)ck, sm);
    if (e != cudaSuccess) return e;
    ck<<<1, 1024, sm, st>>>(sitemajor, M, K, wN, absperm, in_smem ? nullptr : scratch, stage ? 1 : 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (M <= 0) return cudaSuccess;
    sm = refpbwt_fill_smem(K, wN);
    if ((e = ensure_dynamic_smem((const void *)refpbwt_fill_kernel, sm)) !=
        cudaSuccess)
        return e;
    refpbwt_fill_kernel<<<(M + RP_CK - 1) / RP_CK, 1024, sm, st>>>(sitemajor, M, K, wN, compr, absperm, count0);
    return cudaGetLastError();
}

cudaError_t launch_gather_rows(const uint64_t *src, size_t ldsrc, const int64_t *idx, int n, int w, uint64_t *dst,
                               cudaStream_t st) {
    const long tot = (long)n * w;
    if (tot == 0) return cudaSuccess;
    gather_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(src, ldsrc, idx, n, w, dst);
    return cudaGetLastError();
}

cudaError_t launch_transpose(const uint64_t *src, size_t rows, size_t srcw, uint64_t *dst, size_t cols, size_t dstw,
                             cudaStream_t st) {
    return launch_transpose_ld(src, rows, srcw, dst, cols, dstw, dstw, st);
}

cudaError_t launch_transpose_ld(const uint64_t *src, size_t rows, size_t src_ld, uint64_t *dst, size_t cols,
                                size_t dstw, size_t dst_ld, cudaStream_t st) {
    if (!rows || !cols) return cudaSuccess;
    const size_t gy = (cols + 63) / 64;
    if (gy > 65535 || gy > src_ld) return cudaErrorInvalidValue;
    dim3 grid((unsigned)((rows + 63) / 64), (unsigned)gy);
    transpose_kernel<<<grid, 64, 0, st>>>(src, rows, src_ld, dst, cols, dstw, dst_ld);
    return cudaGetLastError();
}

template <class Smem, class Kern, class... Extra>
static cudaError_t smm_launch(Kern kern, int warps, const uint32_t *compr, const int32_t *count0, int M, int K,
                              const uint64_t *phased, int wM, const uint8_t *gt, int nhaps, const int32_t *hapmap,
                              int setmaxerrors, int4 *matches, int cap, int *nmatch, uint32_t *status,
                              cudaStream_t st, Extra... extra) {
    const size_t sm = sizeof(Smem) * warps;
    cudaError_t e = ensure_dynamic_smem((const void *)kern, sm);
    if (e != cudaSuccess) return e;
    const int blocks = (nhaps + warps - 1) / warps;
    kern<<<blocks, warps * 32, sm, st>>>(compr, count0, M, K, phased, wM, gt, nhaps, hapmap, setmaxerrors, matches,
                                        cap, nmatch, status, extra...);
    return cudaGetLastError();
}

size_t smm_gpool_slot_bytes(int K) {
    return K <= 65536 ? sizeof(SmmWarpSmemC<SMM_NODES_RETRY, uint16_t>) : sizeof(SmmWarpSmemC<SMM_NODES_RETRY, int>);
}

template <typename IV>
static cudaError_t launch_smm_compact(const uint32_t *compr, const int32_t *count0, int M, int K,
                                      const uint64_t *phased, int wM, const uint8_t *gt, int nhaps,
                                      const int32_t *hapmap, int setmaxerrors, int4 *matches, int cap, int *nmatch,
                                      uint32_t *status, int warps, void *gpool, int gpool_slots, int *gpool_next,
                                      cudaStream_t st) {
    using Small = SmmWarpSmemC<SMM_NODES, IV>;
    using Big = SmmWarpSmemC<SMM_NODES_RETRY, IV>;
    Big *gp = static_cast<Big *>(gpool);
    cudaError_t e;
    // warps per CTA of the first pass: 1, 2 or 4
    if (warps == 1)
        e = smm_launch<Small>(smm_compact_kernel<SMM_NODES, 1, false, IV>, 1, compr, count0, M, K, phased, wM, gt,
                              nhaps, hapmap, setmaxerrors, matches, cap, nmatch, status, st, gp, gpool_slots,
                              gpool_next);
    else if (warps == 4)
        e = smm_launch<Small>(smm_compact_kernel<SMM_NODES, 4, false, IV>, 4, compr, count0, M, K, phased, wM, gt,
                              nhaps, hapmap, setmaxerrors, matches, cap, nmatch, status, st, gp, gpool_slots,
                              gpool_next);
    else
        e = smm_launch<Small>(smm_compact_kernel<SMM_NODES, SMMC_WARPS, false, IV>, SMMC_WARPS, compr, count0, M, K,
                              phased, wM, gt, nhaps, hapmap, setmaxerrors, matches, cap, nmatch, status, st, gp,
                              gpool_slots, gpool_next);
    if (e != cudaSuccess) return e;
    return smm_launch<Big>(smm_compact_kernel<SMM_NODES_RETRY, 1, true, IV>, 1, compr, count0, M, K, phased, wM, gt,
                           nhaps, hapmap, setmaxerrors, matches, cap, nmatch, status, st, (Big *)nullptr, 0,
                           (int *)nullptr);
}

cudaError_t launch_smm(const uint32_t *compr, const int32_t *count0, int M, int K, const uint64_t *phased, int wM,
                       const uint8_t *gt, int nhaps, const int32_t *hapmap, int setmaxerrors, int4 *matches, int cap,
                       int *nmatch, uint32_t *status, int warps, void *gpool, int gpool_slots, int *gpool_next,
                       cudaStream_t st) {
    if (M < 65536) {   // depths fit the compact tree; interval bounds in 16 bits up to 65,536 haplotypes
        if (K <= 65536)
            return launch_smm_compact<uint16_t>(compr, count0, M, K, phased, wM, gt, nhaps, hapmap, setmaxerrors,
                                                matches, cap, nmatch, status, warps, gpool, gpool_slots, gpool_next,
                                                st);
        return launch_smm_compact<int>(compr, count0, M, K, phased, wM, gt, nhaps, hapmap, setmaxerrors, matches, cap,
                                       nmatch, status, warps, gpool, gpool_slots, gpool_next, st);
    }
    cudaError_t e = smm_launch<SmmWarpSmem<SMM_NODES>>(smm_kernel<SMM_NODES, SMM_WARPS, false>, SMM_WARPS, compr,
                                                       count0, M, K, phased, wM, gt, nhaps, hapmap, setmaxerrors,
                                                       matches, cap, nmatch, status, st);
    if (e != cudaSuccess) return e;
    return smm_launch<SmmWarpSmem<SMM_NODES_RETRY>>(smm_kernel<SMM_NODES_RETRY, 1, true>, 1, compr, count0, M, K,
                                                    phased, wM, gt, nhaps, hapmap, setmaxerrors, matches, cap, nmatch,
                                                    status, st);
}

template <int SPAN>
static void *dosage_kernel_for(bool wide) {
    return wide ? (void *)dosage_kernel<true, SPAN> : (void *)dosage_kernel<false, SPAN>;
}

cudaError_t launch_dosage(const int4 *matches, int cap, const int *nmatch, const int32_t *absperm, int K,
                          const int32_t *refmap, const uint64_t *hapmajor_full, int wMref, const int2 *sinfo,
                          const uint64_t *phased, int wM, const uint8_t *gt, int M, int nhaps, const int32_t *hapmap,
                          int mref_begin, int nsites, int imputeCalls, float *dos, int ldd, uint64_t *bits, int ldb,
                          int span, cudaStream_t st) {
    if (span != 4 && span != 16) span = DOS_SPAN;
    const long ntiles = (nsites + 63) / 64;
    long warps = (long)nhaps * ((ntiles + span - 1) / span);
    long blocks = (warps + 7) / 8;
    const bool wide = M >= 131071;
    using Kern = decltype(&dosage_kernel<false, DOS_SPAN>);
    const Kern kern = (Kern)(span == 4 ? dosage_kernel_for<4>(wide)
                                       : span == 16 ? dosage_kernel_for<16>(wide) : dosage_kernel_for<DOS_SPAN>(wide));
    kern<<<(unsigned)blocks, 256, 0, st>>>(matches, cap, nmatch, absperm, K, refmap, hapmajor_full, wMref, sinfo,
                                           phased, wM, gt, M, nhaps, hapmap, mref_begin, nsites, imputeCalls, dos, ldd,
                                           bits, ldb);
    return cudaGetLastError();
}

cudaError_t launch_segmap(const int64_t *typed, int M, int Mref, const float *af, int nrefhaps_total, int32_t *segm,
                          uint8_t *common, int2 *sinfo, cudaStream_t st) {
    segmap_kernel<<<(Mref + 255) / 256, 256, 0, st>>>(typed, M, Mref, af, nrefhaps_total, segm, common, sinfo);
    return cudaGetLastError();
}

}  // namespace eimp
