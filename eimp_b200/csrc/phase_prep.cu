// Phasing preparation, condensed reference and PBWT kernels for B200 (sm_100a).
//
//  hamming_kernel     -- the Hamming counts of GenotypeVector::compare_withPreInit
//                        (Datatypes.cpp:107-116), 8 targets x 512 reference
//                        haplotypes per CTA.
//  besthaps_kernel    -- Target::findBestHaps (Target.cpp:779-875): exact
//                        K-smallest selection by (errors, index) via a
//                        threshold search.
//  monos_calls_kernel -- Target::findMonos + findCallLocs (Target.cpp:878-950)
//  cref_kernel        -- Target::condensedReferenceT (Target.cpp:953-1059),
//                        one lane per selected haplotype (haplotype-major).
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
// ---------------------------------------------------------------------------
// Hamming counts of GenotypeVector::compare_withPreInit (Datatypes.cpp:107-116)
// for TB targets at once: nerr[t][h] = popc((is0_t & h) | (is2_t & ~h))
// over the typed-site words.  A warp takes one reference haplotype at a time
// and its lanes read the haplotype's row word by word (coalesced); every word
// read serves the CTA's TB targets, whose genotype words sit in shared
// memory (16 * TB * W(M) bytes), so the panel is read once per TB targets
// instead of once per target.  TB is 8 where that fits the shared memory,
// else 4, 2 or 1.  Excluded haplotypes (the target's own in iterations after the
// first, haploid placeholders) get 0xffffffff: never selected.
// ---------------------------------------------------------------------------
constexpr int HAM_WARPS = 8;     // warps per CTA
constexpr int HAM_HPW = 64;      // haplotypes per warp (a CTA builds its targets' genotype words once for 512)
constexpr int HAM_HU = 4;        // haplotypes per pass over the typed-site words

// Reduce-scatter of N (a power of two <= 32) per-lane counts: afterwards v[0]
// of lane l holds the warp's total of count l % N.  Each step halves the
// counts a lane keeps, swapping the other half with the lane that keeps them
// (31 shuffles for N = 32 instead of 32 x 5 for separate reductions).
template <int N>
__device__ __forceinline__ void warp_reduce_scatter(uint32_t (&v)[N], int lane) {
#pragma unroll
    for (int half = N / 2; half >= 1; half >>= 1) {
        const bool up = (lane & half) != 0;
#pragma unroll
        for (int i = 0; i < half; i++) {
            const uint32_t keep = up ? v[half + i] : v[i];
            const uint32_t give = up ? v[i] : v[half + i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, give, half);
        }
    }
#pragma unroll
    for (int o = N; o < 32; o <<= 1) v[0] += __shfl_xor_sync(0xffffffffu, v[0], o);
}

template <int HAM_TB>
__global__ void __launch_bounds__(32 * HAM_WARPS) hamming_kernel(const uint8_t *__restrict__ gt, int ntgt, int M,
                                                                 const uint64_t *__restrict__ hapmajor, int nhaps,
                                                                 int wM, uint32_t *__restrict__ nerr, int self0,
                                                                 const uint8_t *__restrict__ haploid) {
    extern __shared__ uint64_t shm[];
    uint64_t *is0 = shm, *is2 = shm + (size_t)HAM_TB * wM;   // [target][word]
    const int tb = blockIdx.x * HAM_TB;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // genotype bit-planes of the CTA's targets, one 64-site word per warp
    // step: two coalesced byte loads per lane and four ballots
    for (int i = warp; i < HAM_TB * wM; i += HAM_WARPS) {
        const int tt = i / wM, w = i - tt * wM, t = tb + tt;
        uint32_t a[2], b[2];
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int m = w * 64 + half * 32 + lane;
            const uint8_t c = (t < ntgt && m < M) ? gt[(size_t)t * M + m] : 1;   // 1 sets neither plane
            a[half] = __ballot_sync(0xffffffffu, c == 0 || c == 3);
            b[half] = __ballot_sync(0xffffffffu, c == 2 || c == 3);
        }
        if (lane == 0) {
            is0[i] = a[0] | (uint64_t)a[1] << 32;
            is2[i] = b[0] | (uint64_t)b[1] << 32;
        }
    }
    __syncthreads();
    // HAM_HU haplotypes at a time: their rows' words are independent loads
    // in flight together, and each genotype word read from shared memory
    // serves all of them
    constexpr int NV = HAM_HU * HAM_TB;
    const int h0 = (blockIdx.y * HAM_WARPS + warp) * HAM_HPW;
    for (int k = 0; k < HAM_HPW; k += HAM_HU) {
        const int hb = h0 + k;
        if (hb >= nhaps) break;
        uint32_t acc[NV];
#pragma unroll
        for (int i = 0; i < NV; i++) acc[i] = 0;
        for (int w = lane; w < wM; w += 32) {
            uint64_t x[HAM_HU];
#pragma unroll
            for (int u = 0; u < HAM_HU; u++) x[u] = hb + u < nhaps ? hapmajor[(size_t)(hb + u) * wM + w] : 0ull;
#pragma unroll
            for (int q = 0; q < HAM_TB; q++) {
                const uint64_t a = is0[q * wM + w], b = is2[q * wM + w];
#pragma unroll
                for (int u = 0; u < HAM_HU; u++) acc[u * HAM_TB + q] += __popcll((a & x[u]) | (b & ~x[u]));
            }
        }
        // lane l ends with the warp total of count l % NV: haplotype hb + u,
        // target tb + q for l = u * HAM_TB + q
        warp_reduce_scatter<NV>(acc, lane);
        const int u = (lane % NV) / HAM_TB, q = lane % HAM_TB;
        const int h = hb + u, t = tb + q;
        if (lane < NV && h < nhaps && t < ntgt) {
            const int ign = self0 >= 0 ? 2 * (self0 + t) : -2;
            const bool excl = h == ign || h == ign + 1 || (haploid && (h & 1) && haploid[h >> 1]);
            nerr[(size_t)t * nhaps + h] = excl ? 0xffffffffu : acc[0];
        }
    }
}

// haploid: per reference sample, 1 = haploid (null: all diploid).  The
// second column of a haploid sample is never chosen (Target.cpp:800-806,
// 830-838), nor are the target's own two in iterations after the first.
// The error counts come from hamming_kernel.
__global__ void __launch_bounds__(512) besthaps_kernel(const uint8_t *__restrict__ gt, int M,
                                                      const uint64_t *__restrict__ hapmajor, int nhaps, int wM,
                                                      int K, uint32_t *__restrict__ nerr_scratch,
                                                      int32_t *__restrict__ besthaps, uint64_t *__restrict__ flags,
                                                      int wN, int self0, const uint8_t *__restrict__ haploid) {
    __shared__ int buf[32];
    const int t = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    uint32_t *nerr = nerr_scratch + (size_t)t * nhaps;
    int32_t *bh = besthaps + (size_t)t * K;
    uint64_t *fl = flags + (size_t)t * wN;
    for (int w = tid; w < wN; w += nt) fl[w] = 0ull;
    // phasing iterations after the first: the panel ends with the phased
    // targets and a target ignores its own two haplotypes (Target.cpp:791-796)
    const int ign = self0 >= 0 ? 2 * (self0 + t) : -2;
    if (haploid) {
        // with haploid samples: all existing haplotypes when K covers them
        // (Target.cpp:798-811), else the K best of them (below)
        int avail = 0;
        for (int h = tid; h < nhaps; h += nt)
            avail += !(h == ign || h == ign + 1 || ((h & 1) && haploid[h >> 1]));
        avail = block_sum_int(avail, buf);
        if (K >= avail) {
            int carry = 0;
            for (int h0 = 0; h0 < nhaps; h0 += nt) {
                const int h = h0 + tid;
                const int sel = h < nhaps && !(h == ign || h == ign + 1 || ((h & 1) && haploid[h >> 1]));
                int tot;
                const int pos = block_exscan_bit(sel, buf, &tot) + carry;
                if (sel && pos < K) bh[pos] = h;
                const unsigned bal = __ballot_sync(0xffffffffu, sel);
                if ((tid & 31) == 0 && h < nhaps) reinterpret_cast<uint32_t *>(fl)[h >> 5] = bal;
                carry += tot;
                __syncthreads();
            }
            return;
        }
    } else if (ign >= 0 && K >= nhaps - 2) {   // all but the target's own (Target.cpp:798-811)
        for (int h = tid; h < nhaps; h += nt)
            if (h != ign && h != ign + 1) bh[h < ign ? h : h - 2] = h;
        __syncthreads();
        for (int w = tid; w < wN; w += nt) {
            int lo = w * 64;
            uint64_t f = lo + 64 <= nhaps ? ~0ull : (lo >= nhaps ? 0ull : ((1ull << (nhaps - lo)) - 1));
            for (int j = ign; j <= ign + 1; j++)
                if (j >= lo && j < lo + 64) f &= ~(1ull << (j - lo));
            fl[w] = f;
        }
        return;
    }
    if (!haploid && K >= nhaps) {
        for (int h = tid; h < nhaps; h += nt) bh[h] = h;
        __syncthreads();
        for (int w = tid; w < wN; w += nt) {
            int lo = w * 64;
            fl[w] = lo + 64 <= nhaps ? ~0ull : (lo >= nhaps ? 0ull : ((1ull << (nhaps - lo)) - 1));
        }
        return;
    }
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
                            uint32_t *nerr_scratch, int32_t *besthaps, uint64_t *flags, int wN, int self0,
                            const uint8_t *haploid, cudaStream_t st) {
    // the Hamming counts are needed only when K leaves a choice (the kernel
    // below takes every existing haplotype otherwise, without them)
    const int excl = (self0 >= 0 ? 2 : 0);
    if (haploid || K < nhaps - excl) {
        int dev = 0, optin = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if (e != cudaSuccess) return e;
        const size_t per = (size_t)2 * wM * sizeof(uint64_t);   // one target's genotype words
        const int tb = per * 8 <= (size_t)optin ? 8 : per * 4 <= (size_t)optin ? 4 : per * 2 <= (size_t)optin ? 2 : 1;
        const size_t sm = per * tb;
        auto kern = tb == 8 ? hamming_kernel<8> : tb == 4 ? hamming_kernel<4> : tb == 2 ? hamming_kernel<2>
                                                                                        : hamming_kernel<1>;
        if ((e = ensure_dynamic_smem((const void *)kern, sm)) != cudaSuccess)
            return e;
        dim3 grid((unsigned)((ntgt + tb - 1) / tb),
                  (unsigned)((nhaps + HAM_WARPS * HAM_HPW - 1) / (HAM_WARPS * HAM_HPW)));
        kern<<<grid, 32 * HAM_WARPS, sm, st>>>(gt, ntgt, M, hapmajor, nhaps, wM, nerr_scratch, self0, haploid);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    besthaps_kernel<<<ntgt, 512, 0, st>>>(gt, M, hapmajor, nhaps, wM, K, nerr_scratch, besthaps, flags, wN, self0,
                                          haploid);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) monos_calls_kernel(
    const uint8_t *__restrict__ gt, int M, const uint64_t *__restrict__ hapmajor, int wM,
    const int32_t *__restrict__ besthaps, int K, const float *__restrict__ cm, float cMmaxsplit,
    uint64_t *__restrict__ monos, int32_t *__restrict__ splits, int32_t *__restrict__ calls,
    float *__restrict__ cmdiffs, int32_t *__restrict__ nsplits, int32_t *__restrict__ ncalls,
    const uint8_t *__restrict__ tgt_haploid) {
    extern __shared__ unsigned long long smo[];
    unsigned long long *sand = smo, *sor = smo + wM;
    const int t = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
    if (tgt_haploid && tgt_haploid[t]) {   // not phased (Target.cpp:166-203): no split sites
        if (tid == 0) { nsplits[t] = 0; ncalls[t] = 0; }
        return;
    }
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
    if (tid >= 32) return;
    // Target.cpp:900-950, by one warp over 32 sites at a time.  From the
    // first heterozygous site on, a site that is not monomorphic and not
    // missing splits when it is heterozygous (a call) or when it lies more
    // than cMmaxsplit after the previous split.  Heterozygous splits need no
    // order; a homozygous one depends on the split before it, so within the
    // chunk the first homozygous site that passes against the splits known so
    // far is a split, and the sites after it are tested again (such splits
    // are rare: one pass per chunk usually finds none).
    const unsigned FULL = 0xffffffffu;
    const int lane = tid;
    const unsigned lt = (1u << lane) - 1u;
    const uint8_t *g = gt + (size_t)t * M;
    int32_t *sp = splits + (size_t)t * M, *cl = calls + (size_t)t * M;
    float *cd = cmdiffs + (size_t)t * (M + 1);
    int S = 0, C = 0;
    float last = cm[0];
    int m0 = M;   // the first heterozygous site (Target.cpp:905)
    for (int b = 0; b < M; b += 32) {
        const unsigned f = __ballot_sync(FULL, b + lane < M && g[b + lane] == 1);
        if (f) { m0 = b + __ffs((int)f) - 1; break; }
    }
    for (int b = m0; b < M; b += 32) {
        const int m = b + lane;
        const uint8_t c = m < M ? g[m] : 3;
        const bool mono = m < M && ((sand[m >> 6] >> (m & 63)) & 1ull);
        const float cmv = m < M ? cm[m] : 0.0f;
        const bool het = !mono && c == 1, hom = !mono && c != 1 && c != 3;
        const unsigned hets = __ballot_sync(FULL, het);
        unsigned spl = hets;   // the chunk's splits known so far
        int front = -1;        // sites up to here are settled
        for (;;) {
            const unsigned before = spl & lt;
            const int src = before ? 31 - __clz((int)before) : 0;
            const float prev = __shfl_sync(FULL, cmv, src);
            const float lastv = before ? prev : last;
            const bool pass = hom && lane > front && __fsub_rn(cmv, lastv) > cMmaxsplit;
            const unsigned pm = __ballot_sync(FULL, pass);
            if (!pm) break;
            front = __ffs((int)pm) - 1;
            spl |= 1u << front;
        }
        const bool isspl = (spl >> lane) & 1u;
        const int si = S + __popc(spl & lt);
        if (isspl) sp[si] = m;
        if (het) cl[C + __popc(hets & lt)] = si;
        if (spl) last = __shfl_sync(FULL, cmv, 31 - __clz((int)spl));
        S += __popc(spl);
        C += __popc(hets);
    }
    if (S == 0 || C == 0) {   // Target.cpp:923-932
        if (lane == 0) { nsplits[t] = 0; ncalls[t] = 0; }
        return;
    }
    __syncwarp();   // the warp's split and call entries are visible to all its lanes
    S = cl[C - 1] + 1;
    for (int i = lane; i <= S; i += 32) {
        const float a = i < S ? cm[sp[i]] : cm[M - 1];
        const float p = i > 0 ? cm[sp[i - 1]] : cm[0];
        cd[i] = __fsub_rn(a, p);
    }
    if (lane == 0) { nsplits[t] = S; ncalls[t] = C; }
}

cudaError_t launch_monos_calls(const uint8_t *gt, int ntgt, int M, const uint64_t *hapmajor, int wM,
                               const int32_t *besthaps, int K, const float *cm, float cMmaxsplit, uint64_t *monos,
                               int32_t *splits, int32_t *calls, float *cmdiffs, int32_t *nsplits, int32_t *ncalls,
                               const uint8_t *tgt_haploid, cudaStream_t st) {
    size_t sm = (size_t)2 * wM * sizeof(uint64_t);
    if (sm > 48 * 1024) {
        cudaError_t e = ensure_dynamic_smem((const void *)monos_calls_kernel, sm);
        if (e != cudaSuccess) return e;
    }
    monos_calls_kernel<<<ntgt, 256, sm, st>>>(gt, M, hapmajor, wM, besthaps, K, cm, cMmaxsplit, monos, splits, calls,
                                              cmdiffs, nsplits, ncalls, tgt_haploid);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Haploid targets (Target.cpp:166-203, with missing genotypes left missing,
// the default without --impMissing): no phasing; the maternal haplotype and
// dosage are the genotypes (HomAlt -> 1), the paternal outputs are zero, the
// confidence and the call sites count the non-missing sites.  A heterozygous
// genotype is an error.  One CTA per target; diploid targets return at once.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) haploid_phase_kernel(
    const uint8_t *__restrict__ gt, int M, int wM, const uint8_t *__restrict__ tgt_haploid,
    uint64_t *__restrict__ mats, uint64_t *__restrict__ pats, float *__restrict__ dmat, float *__restrict__ dpat,
    float *__restrict__ totalconf, int32_t *__restrict__ ncallsites, uint32_t *__restrict__ status) {
    __shared__ int buf[32];
    const int t = blockIdx.x, tid = threadIdx.x;
    if (!tgt_haploid[t]) return;
    const uint8_t *g = gt + (size_t)t * M;
    int miss = 0, het = 0;
    for (int m = tid; m < M; m += blockDim.x) {
        const uint8_t c = g[m];
        miss += c == 3;
        het |= c == 1;
        dmat[(size_t)t * M + m] = c == 2 ? 1.0f : 0.0f;
        dpat[(size_t)t * M + m] = 0.0f;
    }
    for (int w = tid; w < wM; w += blockDim.x) {
        uint64_t x = 0;
        for (int j = 0; j < 64; j++) {
            const int m = w * 64 + j;
            if (m < M && g[m] == 2) x |= 1ull << j;
        }
        mats[(size_t)t * wM + w] = x;
        pats[(size_t)t * wM + w] = 0ull;
    }
    if (__syncthreads_or(het) && tid == 0) atomicOr(status, (uint32_t)EIMP_ERR_HAPLOID_HET);
    miss = block_sum_int(miss, buf);
    if (tid == 0) {
        totalconf[t] = (float)(M - miss);
        ncallsites[t] = M - miss;
    }
}

cudaError_t launch_haploid_phase(const uint8_t *gt, int ntgt, int M, int wM, const uint8_t *tgt_haploid,
                                 uint64_t *mats, uint64_t *pats, float *dmat, float *dpat, float *totalconf,
                                 int32_t *ncallsites, uint32_t *status, cudaStream_t st) {
    haploid_phase_kernel<<<ntgt, 256, 0, st>>>(gt, M, wM, tgt_haploid, mats, pats, dmat, dpat, totalconf, ncallsites,
                                               status);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Columns of a bit matrix gathered by a map: dst row r bit j = src row r bit
// map[j] (j < ncols; the padding words are zero).  The imputation reference
// without the placeholder column of its haploid samples (PBWTImputer.cpp:67-114).
//
// The reference writes a diploid sample's two columns with one call that
// sets bits pos and pos+1 inside the word of pos (BooleanVector::
// setPairWithPreInit, Datatypes.h:190-197, meant for even pos).  After a
// haploid sample pos can be odd; at pos % 64 == 63 the second bit (2 << 63)
// falls off the word, so that sample's second haplotype reads as all zeros in
// the PBWT.  The kernel reproduces it: a second haplotype (odd panel column)
// whose compacted column starts a word is left zero.  Only the PBWT sees it;
// the dosages read the panel itself (TargetImp.cpp:536).
// ---------------------------------------------------------------------------
__global__ void compact_cols_kernel(const uint64_t *__restrict__ src, int rows, int srcw,
                                    const int32_t *__restrict__ map, int ncols, uint64_t *__restrict__ dst, int dstw) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)rows * dstw) return;
    const int r = (int)(i / dstw), w = (int)(i % dstw);
    const uint64_t *s = src + (size_t)r * srcw;
    uint64_t o = 0;
    for (int j = 0; j < 64; j++) {
        const int c = w * 64 + j;
        if (c < ncols) {
            const int col = map[c];
            if (j == 0 && (col & 1)) continue;   // lost off the previous word (see above)
            o |= ((s[col >> 6] >> (col & 63)) & 1ull) << j;
        }
    }
    dst[i] = o;
}

cudaError_t launch_compact_cols(const uint64_t *src, int rows, int srcw, const int32_t *map, int ncols, uint64_t *dst,
                                int dstw, cudaStream_t st) {
    const long n = (long)rows * dstw;
    compact_cols_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, rows, srcw, map, ncols, dst, dstw);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Target::condensedReferenceT (Target.cpp:953-1059): the condensed reference of
// a target has 2S+1 rows of K bits, one column per selected reference
// haplotype (in besthaps order; identity when K == nhaps, Target.cpp:969-974).
// Row 2j holds the inconsistency of each haplotype over the sites between
// split j-1 and split j (a homozygous target genotype the haplotype does not
// carry), row 2j+1 the haplotype's allele at split site j, row 2S the
// inconsistency after the last split.
//
// Haplotype-major: lane = column.  A lane walks its haplotype's row of the
// haplotype-major reference word by word, once: the split sites of the
// target are a bit mask, so within a word every split closes the running
// segment (its inconsistency row, then the split site's allele row) and the
// rest of the word opens the next one.  One 64-bit addition per word gives
// the inconsistency of every segment the word closes (a carry per segment,
// below), so a split costs two ballots.  The warp's ballot is the 32-bit word
// of an output row.  Grid: (target, 8 output words of 32 columns per CTA);
// the columns past K are written as zero padding up to W(K) words.
// ---------------------------------------------------------------------------
constexpr int CREF_WARPS = 8;

__global__ void __launch_bounds__(32 * CREF_WARPS) cref_kernel(
    const uint8_t *__restrict__ gt, int M, const uint64_t *__restrict__ hapmajor, int wM, int nhaps,
    const int32_t *__restrict__ besthaps, int K, const int32_t *__restrict__ splits,
    const int32_t *__restrict__ nsplits, const int64_t *__restrict__ rowoff, uint64_t *__restrict__ cref,
    const int *__restrict__ skip) {
    if (skip && *skip) return;   // the batch exceeds the reserved rows
    extern __shared__ uint64_t sm[];
    // the target's homozygous genotypes and its split sites as bit masks
    uint64_t *is0 = sm, *is2 = sm + wM, *ssp = sm + 2 * wM;
    const int t = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint8_t *g = gt + (size_t)t * M;
    const int S = nsplits[t];
    const int32_t *sp = splits + (size_t)t * M;
    for (int w = tid; w < wM; w += blockDim.x) {
        uint64_t a = 0, b = 0;
        const int m0 = w * 64;
        for (int j = 0; j < 64 && m0 + j < M; j++) {
            const uint8_t c = g[m0 + j];
            a |= (uint64_t)(c == 0) << j;
            b |= (uint64_t)(c == 2) << j;
        }
        is0[w] = a; is2[w] = b; ssp[w] = 0ull;
    }
    __syncthreads();
    for (int j = tid; j < S; j += blockDim.x) atomicOr((unsigned long long *)&ssp[sp[j] >> 6], 1ull << (sp[j] & 63));
    __syncthreads();
    const int wK = (int)eimp_W(K);
    const int col32 = blockIdx.y * CREF_WARPS + warp;   // 32-bit word of the output rows
    if (col32 >= 2 * wK) return;
    const int k = col32 * 32 + lane;
    const bool valid = k < K;
    const int h = valid ? (K == nhaps ? k : besthaps[(size_t)t * K + k]) : 0;
    const uint64_t *hm = hapmajor + (size_t)h * wM;
    const size_t rstride = 2 * (size_t)wK;   // 32-bit words per row
    uint32_t *out = reinterpret_cast<uint32_t *>(cref + (size_t)rowoff[t] * wK) + col32;
    unsigned open = 0u;   // inconsistency of the open segment (0 or 1)
    uint32_t *o = out;    // the next row pair
    uint64_t hw = valid ? hm[0] : 0ull;
    for (int q = 0; q < wM; q++) {
        const uint64_t a = hw;
        if (q + 1 < wM) hw = valid ? hm[q + 1] : 0ull;   // next word in flight
        const uint64_t s = ssp[q];
        const uint64_t x = (a & is0[q]) | (~a & is2[q]);
        // One addition closes every segment of the word: ~s has ones at the
        // positions that are not split sites, so adding the inconsistencies
        // there (and the open segment's state at bit 0) carries out of each
        // segment that holds one into the split site that closes it, and no
        // carry crosses a split site.  The carry out of the word is the state
        // of the segment left open after the word's last split.
        const uint64_t ns = ~s;
        const uint64_t t = ns + (x & ns);
        const uint64_t r = t + (uint64_t)open;
        open = (t < ns || r < t) ? 1u : 0u;
        const uint64_t marks = valid ? r & s : 0ull;
#pragma unroll
        for (int hf = 0; hf < 2; hf++) {
            uint32_t bnd = (uint32_t)(s >> (32 * hf));
            const uint32_t mk = (uint32_t)(marks >> (32 * hf)), al = (uint32_t)(a >> (32 * hf));
            while (bnd) {
                const int b = __ffs((int)bnd) - 1;
                const unsigned wi = __ballot_sync(0xffffffffu, (mk >> b) & 1u);
                const unsigned ws = __ballot_sync(0xffffffffu, (al >> b) & 1u);
                if (lane == 0) { o[0] = wi; o[rstride] = ws; }
                o += 2 * rstride;
                bnd &= bnd - 1;
            }
        }
    }
    const unsigned wi = __ballot_sync(0xffffffffu, valid && open);
    if (lane == 0) o[0] = wi;
}

cudaError_t launch_cref(const uint8_t *gt, int ntgt, int M, const uint64_t *hapmajor, int wM, int nhaps,
                        const int32_t *besthaps, int K, const int32_t *splits, const int32_t *nsplits,
                        const int64_t *rowoff, uint64_t *cref, const int *skip, cudaStream_t st) {
    const size_t sm = (size_t)3 * wM * sizeof(uint64_t);
    if (sm > 48 * 1024) {
        cudaError_t e = ensure_dynamic_smem((const void *)cref_kernel, sm);
        if (e != cudaSuccess) return e;
    }
    const int wK = (int)eimp_W(K);
    dim3 grid((unsigned)ntgt, (unsigned)((2 * wK + CREF_WARPS - 1) / CREF_WARPS));
    cref_kernel<<<grid, 32 * CREF_WARPS, sm, st>>>(gt, M, hapmajor, wM, nhaps, besthaps, K, splits, nsplits, rowoff,
                                                   cref, skip);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// PBWT::buildComprPBWT (PBWT.cpp:207-285) of each target's condensed
// reference, forward and backward (rows in sweep order), one CTA per (target,
// direction).  Each thread owns WPT consecutive 32-position words of the
// prefix order.  Per row: the thread gathers its words' bits in the current
// prefix order (a word is the row format's data word, the tail padded with
// ones) and counts their zeros; one block scan gives every word's zeros
// before it; the thread writes its [data, zeros through the word] pairs and
// places its haplotypes in the next prefix order (zeros first, stable).  The
// prefix arrays are 16-bit (K <= 65536) and XOR-swizzled within each 32-entry
// block, so that the 32 lanes reading the same pair of positions of their own
// words hit 32 different banks.  A thread reads its words' haplotypes once
// per row, sixteen 32-bit pairs per word, and keeps them in registers from
// the gather to the placement.  The next row is copied into shared memory asynchronously
// while the current one is processed.  The forward CTA also writes each
// row's zero count.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// position p of the prefix order -> its slot in the swizzled array
__device__ __forceinline__ int pswz(int p) { return p ^ ((p >> 5) & 31); }

// The data word of one 32-position block of the prefix order (key = block &
// 31, the block's swizzle): positions 2i and 2i+1 sit in the 32-bit pair
// i ^ (key >> 1) of the block, swapped when key is odd, so sixteen 32-bit
// loads (the 32 lanes of a warp on 32 different banks) fetch the block.  The
// pairs go to hp in position order; the bits are pushed from position 31
// down to 0.
__device__ __forceinline__ uint32_t pbwt_gather(const uint32_t *__restrict__ pw, int key,
                                                const uint32_t *__restrict__ row, uint32_t hp[16]) {
    const int k2 = key >> 1;
    const unsigned rot = (unsigned)(key & 1) << 4;
    uint32_t b = 0u;
#pragma unroll
    for (int i = 15; i >= 0; i--) {
        const uint32_t v = pw[i ^ k2];
        const uint32_t x = __funnelshift_r(v, v, rot);
        hp[i] = x;
        const uint32_t h0 = x & 0xffffu, h1 = x >> 16;
        const uint32_t r1 = row[h1 >> 5], r0 = row[h0 >> 5];
        b = (b << 1) | (__funnelshift_r(r1, r1, h1) & 1u);
        b = (b << 1) | (__funnelshift_r(r0, r0, h0) & 1u);
    }
    return b;
}

// Places the haplotypes of one block (hp, data word b) in the next prefix
// order: a zero at the next zero place dz, a one at the next one place d1
// (stable).  CHECK: only the first nv positions exist (the block holding K).
template <bool CHECK>
__device__ __forceinline__ void pbwt_place(uint16_t *__restrict__ nperm, const uint32_t hp[16], uint32_t b, int nv,
                                           int &dz, int &d1) {
#pragma unroll
    for (int j = 0; j < 32; j++) {
        if (!CHECK || j < nv) {
            const uint32_t x = hp[j >> 1];
            const uint16_t h = (uint16_t)((j & 1) ? x >> 16 : x & 0xffffu);
            const int one = (int)((b >> j) & 1u);
            nperm[pswz(one ? d1 : dz)] = h;
            d1 += one;
            dz += 1 - one;
        }
    }
}

template <int WPT>
__global__ void __launch_bounds__(1024) pbwt_kernel(const uint64_t *__restrict__ cref,
                                                    const int64_t *__restrict__ rowoff, int K,
                                                    uint32_t *__restrict__ pbwt, size_t rowstride, int emit_padded,
                                                    int32_t *__restrict__ count0, const int *__restrict__ skip) {
    if (skip && *skip) return;   // the batch exceeds the reserved rows
    extern __shared__ __align__(16) uint8_t smem[];
    const int t = blockIdx.x >> 1, dir = blockIdx.x & 1;
    const int wK = (int)eimp_W(K);
    const int nwords = (K + 31) / 32;
    const int nthreads = blockDim.x, nwarps = nthreads >> 5;
    uint64_t *rowbuf = reinterpret_cast<uint64_t *>(smem);                 // 2 x wK
    int *wtot = reinterpret_cast<int *>(rowbuf + 2 * wK);                  // 32
    uint16_t *perm = reinterpret_cast<uint16_t *>(wtot + 32);              // nwords*32, swizzled
    uint16_t *nperm = perm + nwords * 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t r0 = rowoff[t];
    const int Mp = (int)(rowoff[t + 1] - r0);
    const uint64_t *rows = cref + (size_t)r0 * wK;
    uint32_t *out = pbwt + (size_t)(2 * r0 + (dir ? Mp : 0)) * rowstride;
    const int w0 = tid * WPT;                      // the thread's first word
    const int nchunk = wK / 2;                     // 16-byte pieces of a row
    // identity order; the padding positions past K hold haplotype 0 in both
    // arrays (never written later, never used for a bit)
    for (int i = tid; i < nwords * 32; i += nthreads) perm[pswz(i)] = nperm[pswz(i)] = (uint16_t)(i < K ? i : 0);
    if (Mp > 0) {
        const uint64_t *src = rows + (size_t)(dir ? Mp - 1 : 0) * wK;
        for (int c = tid; c < nchunk; c += nthreads) cp_async16(rowbuf + 2 * c, src + 2 * c);
    }
    cp_async_commit();
    for (int midx = 0; midx < Mp; midx++) {
        const int m = dir ? Mp - 1 - midx : midx;
        const uint32_t *row = reinterpret_cast<const uint32_t *>(rowbuf + (midx & 1) * wK);
        cp_async_wait_all();
        __syncthreads();   // this row has landed; the previous row's placements are done
        if (midx + 1 < Mp) {
            const uint64_t *src = rows + (size_t)(dir ? m - 1 : m + 1) * wK;
            uint64_t *dst = rowbuf + ((midx + 1) & 1) * wK;
            for (int c = tid; c < nchunk; c += nthreads) cp_async16(dst + 2 * c, src + 2 * c);
        }
        cp_async_commit();
        // the thread's data words in the current prefix order, and the
        // haplotypes of their positions (two per register, in position order)
        // kept for the placement
        uint32_t word[WPT];
        uint32_t hp[WPT][16];
        int zsum = 0;
#pragma unroll
        for (int q = 0; q < WPT; q++) {
            const int w = w0 + q;
            uint32_t b = ~0u;
            if (w < nwords) {
                b = pbwt_gather(reinterpret_cast<const uint32_t *>(perm + w * 32), w & 31, row, hp[q]);
                const int past = K - w * 32;   // positions past K read as 1 (the row format's padding)
                if (past < 32) b |= ~0u << past;
                zsum += __popc(~b);
            }
            word[q] = b;
        }
        // zeros before the thread's words: warp scan, then the warps' totals
        int inc = zsum;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wtot[warp] = inc;
        __syncthreads();
        int zb = inc - zsum, cnt0 = 0;
        for (int q = 0; q < nwarps; q++) { const int v = wtot[q]; cnt0 += v; if (q < warp) zb += v; }
        uint32_t *o = out + (size_t)midx * rowstride;
#pragma unroll
        for (int q = 0; q < WPT; q++) {
            const int w = w0 + q;
            if (w >= nwords) continue;
            const uint32_t b = word[q];
            // the next zero's place (zeros so far) and the next one's (cnt0 +
            // ones so far)
            int dz = zb, d1 = cnt0 + w * 32 - zb;
            if (w * 32 + 32 <= K) pbwt_place<false>(nperm, hp[q], b, 32, dz, d1);
            else pbwt_place<true>(nperm, hp[q], b, K - w * 32, dz, d1);
            reinterpret_cast<uint2 *>(o)[w] = make_uint2(b, (uint32_t)dz);
            zb = dz;
        }
        if (emit_padded)
            for (size_t jj = 2 * (size_t)nwords + tid; jj < rowstride; jj += nthreads) o[jj] = 0u;
        if (dir == 0 && tid == nthreads - 1) count0[r0 + m] = cnt0;
        uint16_t *tp = perm; perm = nperm; nperm = tp;
    }
    cp_async_wait_all();
}

// shared memory of a CTA: two rows, the warps' zero totals, two prefix arrays
static size_t pbwt_smem(int K) {
    const int nwords = (K + 31) / 32;
    return (size_t)2 * eimp_W(K) * 8 + 32 * 4 + (size_t)2 * nwords * 32 * 2;
}

template <int WPT>
static cudaError_t launch_pbwt_w(const uint64_t *cref, int32_t *count0, const int64_t *rowoff, int ntgt, int K,
                                 uint32_t *pbwt, size_t rowstride, int emit_padded, const int *skip,
                                 cudaStream_t st) {
    const int nwords = (K + 31) / 32;
    const int nthreads = ((nwords + WPT - 1) / WPT + 31) / 32 * 32;
    const size_t sm = pbwt_smem(K);
    cudaError_t e = ensure_dynamic_smem((const void *)pbwt_kernel<WPT>, sm);
    if (e != cudaSuccess) return e;
    pbwt_kernel<WPT><<<2 * ntgt, nthreads, sm, st>>>(cref, rowoff, K, pbwt, rowstride, emit_padded, count0, skip);
    return cudaGetLastError();
}

cudaError_t launch_pbwt(const uint64_t *cref, int32_t *count0, const int64_t *rowoff, int ntgt, int K,
                        uint32_t *pbwt, size_t rowstride, int emit_padded, const int *skip, cudaStream_t st) {
    // the 8-byte pair stores need 8-byte aligned rows
    if (K < 1 || K > 65536 || rowstride % 2) return cudaErrorInvalidValue;
    const int nwords = (K + 31) / 32;
    if (nwords <= 1024) return launch_pbwt_w<1>(cref, count0, rowoff, ntgt, K, pbwt, rowstride, emit_padded, skip, st);
    return launch_pbwt_w<2>(cref, count0, rowoff, ntgt, K, pbwt, rowstride, emit_padded, skip, st);
}

// ---------------------------------------------------------------------------
// Row offsets of the batch's condensed references (the exclusive prefix of
// 2*nsplits+1, GPUHandler.cpp:139-143) computed on the device, so that no
// host round trip sits between the preparation and the condensed reference.
// One CTA: per-thread chunk sums, a block scan, then the chunk prefixes.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) rowoff_kernel(const int32_t *__restrict__ nsplits, int ntgt,
                                                      int64_t *__restrict__ rowoff, int64_t cap, int *__restrict__ skip,
                                                      uint32_t *__restrict__ status) {
    __shared__ long long part[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x;
    const int per = (ntgt + nt - 1) / nt;
    const int lo = min(ntgt, tid * per), hi = min(ntgt, lo + per);
    long long sum = 0;
    for (int t = lo; t < hi; t++) sum += 2 * (long long)nsplits[t] + 1;
    long long inc = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) part[warp] = inc;
    __syncthreads();
    long long base = 0;
    for (int q = 0; q < warp; q++) base += part[q];
    long long run = base + inc - sum;
    for (int t = lo; t < hi; t++) { rowoff[t] = run; run += 2 * (long long)nsplits[t] + 1; }
    if (tid == nt - 1) {
        rowoff[ntgt] = run;
        const int over = run > cap;
        *skip = over;
        if (over) atomicOr(status, (uint32_t)EIMP_ERR_ROWS_OVERFLOW);
    }
}

cudaError_t launch_rowoff(const int32_t *nsplits, int ntgt, int64_t *rowoff, int64_t cap, int *skip,
                          uint32_t *status, cudaStream_t st) {
    rowoff_kernel<<<1, 1024, 0, st>>>(nsplits, ntgt, rowoff, cap, skip, status);
    return cudaGetLastError();
}

}  // namespace eimp
