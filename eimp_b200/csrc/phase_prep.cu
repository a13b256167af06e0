// Phasing preparation, condensed reference and PBWT kernels for B200 (sm_100a).
//
//  besthaps_kernel    -- Target::findBestHaps (Target.cpp:779-875) with the
//                        Hamming count of GenotypeVector::compare_withPreInit
//                        (Datatypes.cpp:107-116); exact K-smallest selection
//                        by (errors, index) via a threshold search.
//  monos_calls_kernel -- Target::findMonos + findCallLocs (Target.cpp:878-950)
//  cref_kernel        -- Target::condensedReferenceT (Target.cpp:953-1059)
//  pbwt_kernel        -- PBWT::buildComprPBWT (PBWT.cpp:207-285), forward and
//                        backward, one CTA per (target, direction).
#include "common.cuh"
#include "kernels.h"

namespace eimp {

__device__ __forceinline__ int block_sum_int(int v, int *buf) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) buf[wid] = v;
    __syncthreads();
    int r = 0;
    for (int i = 0; i < nw; i++) r += buf[i];
    __syncthreads();
    return r;
}

// exclusive prefix of a 0/1 predicate over the block (thread order); returns
// the prefix for this thread, *total gets the block total
__device__ __forceinline__ int block_exscan_bit(int pred, int *buf, int *total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    unsigned b = __ballot_sync(0xffffffffu, pred);
    int within = __popc(b & ((1u << lane) - 1u));
    __syncthreads();
    if (lane == 0) buf[wid] = __popc(b);
    __syncthreads();
    int before = 0, tot = 0;
    for (int i = 0; i < nw; i++) { if (i < wid) before += buf[i]; tot += buf[i]; }
    *total = tot;
    return before + within;
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) besthaps_kernel(const uint8_t *__restrict__ gt, int M,
                                                      const uint64_t *__restrict__ hapmajor, int nhaps, int wM,
                                                      int K, uint32_t *__restrict__ nerr_scratch,
                                                      int32_t *__restrict__ besthaps, uint64_t *__restrict__ flags,
                                                      int wN) {
    extern __shared__ uint64_t sm[];
    uint64_t *is0 = sm, *is2 = sm + wM;
    __shared__ int buf[32];
    const int t = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const uint8_t *g = gt + (size_t)t * M;
    for (int w = tid; w < wM; w += nt) {
        uint64_t a = 0, b = 0;
        for (int j = 0; j < 64; j++) {
            int m = w * 64 + j;
            if (m < M) {
                uint8_t c = g[m];
                if (c == 0 || c == 3) a |= 1ull << j;
                if (c == 2 || c == 3) b |= 1ull << j;
            }
        }
        is0[w] = a; is2[w] = b;
    }
    __syncthreads();
    uint32_t *nerr = nerr_scratch + (size_t)t * nhaps;
    int32_t *bh = besthaps + (size_t)t * K;
    uint64_t *fl = flags + (size_t)t * wN;
    for (int w = tid; w < wN; w += nt) fl[w] = 0ull;
    if (K >= nhaps) {
        for (int h = tid; h < nhaps; h += nt) bh[h] = h;
        __syncthreads();
        for (int w = tid; w < wN; w += nt) {
            int lo = w * 64;
            fl[w] = lo + 64 <= nhaps ? ~0ull : (lo >= nhaps ? 0ull : ((1ull << (nhaps - lo)) - 1));
        }
        return;
    }
    for (int h = tid; h < nhaps; h += nt) {
        const uint64_t *row = hapmajor + (size_t)h * wM;
        uint32_t e = 0;
        for (int w = 0; w < wM; w++) e += __popcll((is0[w] & row[w]) | (is2[w] & ~row[w]));
        nerr[h] = e;
    }
    __syncthreads();
    // smallest threshold thr with #(nerr <= thr) >= K
    int lo = 0, hi = M;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        int c = 0;
        for (int h = tid; h < nhaps; h += nt) c += nerr[h] <= (uint32_t)mid;
        c = block_sum_int(c, buf);
        if (c >= K) hi = mid; else lo = mid + 1;
    }
    const uint32_t thr = (uint32_t)lo;
    int below = 0;
    for (int h = tid; h < nhaps; h += nt) below += nerr[h] < thr;
    below = block_sum_int(below, buf);
    const int need = K - below;   // haps with nerr == thr taken in index order (std::sort of pairs)
    int eqcarry = 0, selcarry = 0;
    for (int h0 = 0; h0 < nhaps; h0 += nt) {
        int h = h0 + tid;
        uint32_t e = h < nhaps ? nerr[h] : 0xffffffffu;
        int iseq = h < nhaps && e == thr;
        int eqtot;
        int eqrank = block_exscan_bit(iseq, buf, &eqtot) + eqcarry;
        int sel = h < nhaps && (e < thr || (iseq && eqrank < need));
        int seltot;
        int pos = block_exscan_bit(sel, buf, &seltot) + selcarry;
        if (sel && pos < K) bh[pos] = h;
        unsigned bal = __ballot_sync(0xffffffffu, sel);
        if ((tid & 31) == 0 && h < nhaps) {
            // h is a multiple of 32 here: write the 32-bit half of the flag word
            reinterpret_cast<uint32_t *>(fl)[h >> 5] = bal;
        }
        eqcarry += eqtot;
        selcarry += seltot;
        __syncthreads();
    }
}

cudaError_t launch_besthaps(const uint8_t *gt, int ntgt, int M, const uint64_t *hapmajor, int nhaps, int wM, int K,
                            uint32_t *nerr_scratch, int32_t *besthaps, uint64_t *flags, int wN, cudaStream_t st) {
    size_t sm = (size_t)2 * wM * sizeof(uint64_t);
    if (sm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(besthaps_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
    }
    besthaps_kernel<<<ntgt, 512, sm, st>>>(gt, M, hapmajor, nhaps, wM, K, nerr_scratch, besthaps, flags, wN);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) monos_calls_kernel(
    const uint8_t *__restrict__ gt, int M, const uint64_t *__restrict__ hapmajor, int wM,
    const int32_t *__restrict__ besthaps, int K, const float *__restrict__ cm, float cMmaxsplit,
    uint64_t *__restrict__ monos, int32_t *__restrict__ splits, int32_t *__restrict__ calls,
    float *__restrict__ cmdiffs, int32_t *__restrict__ nsplits, int32_t *__restrict__ ncalls) {
    extern __shared__ unsigned long long smo[];
    unsigned long long *sand = smo, *sor = smo + wM;
    const int t = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const int32_t *bh = besthaps + (size_t)t * K;
    for (int w = tid; w < wM; w += nt) { sand[w] = ~0ull; sor[w] = 0ull; }
    __syncthreads();
    // AND / OR of the K best haps per word column; mono = all equal
    const int slices = wM >= nt ? 1 : nt / wM;
    for (int w0 = 0; w0 < wM; w0 += nt) {
        int idx = tid;
        int w = w0 + (slices == 1 ? idx : idx % wM);
        int sl = slices == 1 ? 0 : idx / wM;
        if (w < wM && sl < slices) {
            unsigned long long a = ~0ull, o = 0ull;
            for (int k = sl; k < K; k += slices) {
                unsigned long long x = hapmajor[(size_t)bh[k] * wM + w];
                a &= x; o |= x;
            }
            atomicAnd(&sand[w], a);
            atomicOr(&sor[w], o);
        }
    }
    __syncthreads();
    uint64_t *mo = monos + (size_t)t * wM;
    for (int w = tid; w < wM; w += nt) {
        int lo = w * 64;
        uint64_t mask = lo + 64 <= M ? ~0ull : (lo >= M ? 0ull : ((1ull << (M - lo)) - 1));
        uint64_t v = (K <= 1) ? mask : ((sand[w] | ~sor[w]) & mask);
        sand[w] = v;
        mo[w] = v;
    }
    __syncthreads();
    if (tid != 0) return;
    // Target.cpp:900-950 (sequential scan)
    const uint8_t *g = gt + (size_t)t * M;
    int32_t *sp = splits + (size_t)t * M, *cl = calls + (size_t)t * M;
    float *cd = cmdiffs + (size_t)t * (M + 1);
    int S = 0, C = 0;
    float last = cm[0];
    int m = 0;
    for (; m < M; m++) if (g[m] == 1) break;
    for (; m < M; m++) {
        uint8_t c = g[m];
        bool mono = (sand[m >> 6] >> (m & 63)) & 1ull;
        if (!mono && c != 3 && (c == 1 || __fsub_rn(cm[m], last) > cMmaxsplit)) {
            if (c == 1) cl[C++] = S;
            sp[S++] = m;
            last = cm[m];
        }
    }
    if (S == 0 || C == 0) { nsplits[t] = 0; ncalls[t] = 0; return; }   // Target.cpp:923-932
    S = cl[C - 1] + 1;
    cd[0] = __fsub_rn(cm[sp[0]], cm[0]);
    for (int i = 1; i < S; i++) cd[i] = __fsub_rn(cm[sp[i]], cm[sp[i - 1]]);
    cd[S] = __fsub_rn(cm[M - 1], cm[sp[S - 1]]);
    nsplits[t] = S;
    ncalls[t] = C;
}

cudaError_t launch_monos_calls(const uint8_t *gt, int ntgt, int M, const uint64_t *hapmajor, int wM,
                               const int32_t *besthaps, int K, const float *cm, float cMmaxsplit, uint64_t *monos,
                               int32_t *splits, int32_t *calls, float *cmdiffs, int32_t *nsplits, int32_t *ncalls,
                               cudaStream_t st) {
    size_t sm = (size_t)2 * wM * sizeof(uint64_t);
    if (sm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(monos_calls_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
    }
    monos_calls_kernel<<<ntgt, 256, sm, st>>>(gt, M, hapmajor, wM, besthaps, K, cm, cMmaxsplit, monos, splits, calls,
                                              cmdiffs, nsplits, ncalls);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// compact a full-width row (smem) to the K best haps -> dst (wK words)
__device__ int compact_row(const uint64_t *src, int nhaps, const int32_t *bh, int K, int wK, uint64_t *dst,
                           int *buf) {
    int cnt1 = 0;
    if (K == nhaps) {
        int nopad = (nhaps + 63) / 64;
        for (int w = threadIdx.x; w < wK; w += blockDim.x) {
            uint64_t x = 0;
            if (w < nopad) {
                x = src[w];
                if (w == nopad - 1 && (nhaps & 63)) x &= (1ull << (nhaps & 63)) - 1;
            }
            dst[w] = x;
            cnt1 += __popcll(x);
        }
    } else {
        for (int w = threadIdx.x; w < wK; w += blockDim.x) {
            uint64_t x = 0;
            int k0 = w * 64;
            int kn = min(64, K - k0);
            for (int b = 0; b < kn; b++) {
                int h = bh[k0 + b];
                x |= ((src[h >> 6] >> (h & 63)) & 1ull) << b;
            }
            dst[w] = x;
            cnt1 += __popcll(x);
        }
    }
    return K - block_sum_int(cnt1, buf);
}

__global__ void __launch_bounds__(256) cref_kernel(const uint8_t *__restrict__ gt, int M,
                                                  const uint64_t *__restrict__ sitemajor, int nhaps, int wN,
                                                  const int32_t *__restrict__ besthaps, int K,
                                                  const int32_t *__restrict__ splits, const int32_t *__restrict__ nsplits,
                                                  const int64_t *__restrict__ rowoff, uint64_t *__restrict__ cref,
                                                  int32_t *__restrict__ count0) {
    extern __shared__ uint64_t sm[];
    uint64_t *incon = sm, *srow = sm + wN;
    __shared__ int buf[32];
    const int t = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    const int S = nsplits[t];
    const int wK = (int)eimp_W(K);
    const uint8_t *g = gt + (size_t)t * M;
    const int32_t *bh = besthaps + (size_t)t * K;
    const int32_t *sp = splits + (size_t)t * M;
    uint64_t *out = cref + (size_t)rowoff[t] * wK;
    int32_t *c0 = count0 + rowoff[t];
    const int nopad = (nhaps + 63) / 64;
    for (int w = tid; w < wN; w += nt) incon[w] = 0ull;
    __syncthreads();
    int si = 0;
    int next = S > 0 ? sp[0] : -1;
    int row = 0;
    for (int m = 0; m < M; m++) {
        const uint64_t *r = sitemajor + (size_t)m * wN;
        if (m == next) {
            __syncthreads();
            int z = compact_row(incon, nhaps, bh, K, wK, out + (size_t)row * wK, buf);
            if (tid == 0) c0[row] = z;
            row++;
            for (int w = tid; w < wN; w += nt) { incon[w] = 0ull; srow[w] = r[w]; }
            __syncthreads();
            z = compact_row(srow, nhaps, bh, K, wK, out + (size_t)row * wK, buf);
            if (tid == 0) c0[row] = z;
            row++;
            si++;
            next = si < S ? sp[si] : -1;
        } else {
            uint8_t c = g[m];
            if (c == 0) for (int w = tid; w < nopad; w += nt) incon[w] |= r[w];
            else if (c == 2) for (int w = tid; w < nopad; w += nt) incon[w] |= ~r[w];
        }
    }
    __syncthreads();
    int z = compact_row(incon, nhaps, bh, K, wK, out + (size_t)row * wK, buf);
    if (tid == 0) c0[row] = z;
}

cudaError_t launch_cref(const uint8_t *gt, int ntgt, int M, const uint64_t *sitemajor, int nhaps, int wN,
                        const int32_t *besthaps, int K, const int32_t *splits, const int32_t *nsplits,
                        const int64_t *rowoff, uint64_t *cref, int32_t *count0, cudaStream_t st) {
    size_t sm = (size_t)2 * wN * sizeof(uint64_t);
    if (sm > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(cref_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e != cudaSuccess) return e;
    }
    cref_kernel<<<ntgt, 256, sm, st>>>(gt, M, sitemajor, nhaps, wN, besthaps, K, splits, nsplits, rowoff, cref,
                                       count0);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
__device__ void block_exscan_small(int *a, int n, int *warpbuf, int *total) {
    // n <= a few thousand: chunked per-thread sums, then a warp-level scan
    const int tid = threadIdx.x, nt = blockDim.x;
    const int per = (n + nt - 1) / nt;
    const int lo = tid * per, hi = min(n, lo + per);
    int s = 0;
    for (int i = lo; i < hi; i++) s += a[i];
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

__global__ void __launch_bounds__(512) pbwt_kernel(const uint64_t *__restrict__ cref, const int64_t *__restrict__ rowoff,
                                                  int K, uint32_t *__restrict__ pbwt, size_t rowstride,
                                                  int emit_padded) {
    extern __shared__ uint8_t smem[];
    const int t = blockIdx.x >> 1, dir = blockIdx.x & 1;
    const int wK = (int)eimp_W(K);
    const int nwords = (K + 31) / 32;
    int32_t *perm = reinterpret_cast<int32_t *>(smem);
    int32_t *nperm = perm + K;
    uint32_t *row = reinterpret_cast<uint32_t *>(nperm + K);   // 2*wK
    uint32_t *data = row + 2 * wK;                              // nwords
    int *pz = reinterpret_cast<int *>(data + nwords);           // nwords
    int *warpbuf = pz + nwords;                                 // 32
    int *tot = warpbuf + 32;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
    const int64_t r0 = rowoff[t];
    const int Mp = (int)(rowoff[t + 1] - r0);
    const uint64_t *rows = cref + (size_t)r0 * wK;
    uint32_t *out = pbwt + (size_t)(2 * r0 + (dir ? Mp : 0)) * rowstride;
    for (int i = tid; i < K; i += blockDim.x) perm[i] = i;
    __syncthreads();
    for (int midx = 0; midx < Mp; midx++) {
        const int m = dir ? Mp - 1 - midx : midx;
        const uint64_t *src = rows + (size_t)m * wK;
        for (int w = tid; w < wK; w += blockDim.x) {
            uint64_t x = src[w];
            row[2 * w] = (uint32_t)x;
            row[2 * w + 1] = (uint32_t)(x >> 32);
        }
        __syncthreads();
        for (int w = wid; w < nwords; w += nwarps) {
            int i = w * 32 + lane;
            int bit = 1;
            if (i < K) { int h = perm[i]; bit = (row[h >> 5] >> (h & 31)) & 1; }
            uint32_t b = __ballot_sync(0xffffffffu, bit);
            if (lane == 0) { data[w] = b; pz[w] = __popc(~b); }
        }
        __syncthreads();
        block_exscan_small(pz, nwords, warpbuf, tot);
        const int cnt0 = *tot;
        uint32_t *o = out + (size_t)midx * rowstride;
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
            if (lane == 0) { o[2 * w] = b; o[2 * w + 1] = (uint32_t)(zb + __popc(~b)); }
        }
        if (emit_padded)
            for (size_t j = 2 * (size_t)nwords + tid; j < rowstride; j += blockDim.x) o[j] = 0u;
        __syncthreads();
        int32_t *tp = perm; perm = nperm; nperm = tp;
    }
}

cudaError_t launch_pbwt(const uint64_t *cref, const int32_t *count0, const int64_t *rowoff, int ntgt, int K,
                        uint32_t *pbwt, size_t rowstride, int emit_padded, cudaStream_t st) {
    (void)count0;
    const int wK = (int)eimp_W(K), nwords = (K + 31) / 32;
    size_t sm = (size_t)2 * K * 4 + (size_t)2 * wK * 4 + (size_t)nwords * 4 * 2 + 33 * 4;
    cudaError_t e = cudaFuncSetAttribute(pbwt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    pbwt_kernel<<<2 * ntgt, 512, sm, st>>>(cref, rowoff, K, pbwt, rowstride, emit_padded);
    return cudaGetLastError();
}

}  // namespace eimp
