// Per-site output statistics of an imputed bunch (sm_100a).
//
//  site_stats_kernel -- the numeric part of VCFData::writeVCFImputedBunch
//                       (VCFData.cpp:3068-3446): the allele dosage and allele
//                       written for every target haplotype (imputation
//                       conflicts take the reference panel's allele
//                       frequency, typed sites keep the phased call unless
//                       --overwriteCalls / --improveCalls), the optional DS
//                       and GP fields, and per site AC, AN, the dosage AF and
//                       MAF, the minimac4 r2 and whether the record passes the
//                       r2 / MAF output filters; haploid targets write their
//                       first haplotype only; the --improveCalls run
//                       statistics (VCFData.cpp:3306-3330).
//
// A CTA handles 32 sites (one per lane) and walks the targets in chunks of
// SS_CHUNK.  Its SS_PROD producer warps share a chunk's targets: each loads
// the dosages and alleles of its targets for the 32 sites (a warp reads 32
// consecutive floats of a haplotype row: coalesced), applies the
// substitutions, writes the allele dosages, alleles, DS and GP, and leaves
// the per-target float terms (ADS0 + ADS1 and ADS0^2 + ADS1^2) in shared
// memory.  A summing warp adds them into the double sums in target order --
// the reference's order and roundings -- one chunk behind the producers
// (double-buffered terms, one CTA barrier per chunk).  HBM-bound: each site
// reads the 2N dosages and writes the 2N allele dosages.
#include "common.cuh"
#include "kernels.h"

namespace eimp {

constexpr int SS_PROD = 8;                  // producer warps per CTA
constexpr int SS_CHUNK = 64;                // targets per chunk
constexpr int SS_PER = SS_CHUNK / SS_PROD;  // targets of a producer warp per chunk
constexpr int SS_U = 4;                     // targets whose inputs a producer loads ahead

__device__ __forceinline__ float one_minus(float x) {   // `1.0 - x` with x float, rounded back to float
    return (float)__dsub_rn(1.0, (double)x);
}

// htslib's bit patterns for a missing float and the end of a shorter vector
__device__ __forceinline__ float bcf_missing() { return __uint_as_float(0x7F800001u); }
__device__ __forceinline__ float bcf_vector_end() { return __uint_as_float(0x7F800002u); }

template <bool DS, bool GP, bool HAP>
__global__ void __launch_bounds__((SS_PROD + 1) * 32, 3) site_stats_kernel(SiteStatsArgs a) {
    __shared__ float tsum[2][SS_CHUNK][32], tsq[2][SS_CHUNK][32];
    __shared__ int wac[SS_PROD][32], wnv[SS_PROD][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int isite = blockIdx.x * 32 + lane;
    const bool valid = isite < a.nsites;
    const int s = valid ? isite : 0;
    const int mref = a.mref_begin + s;
    const float rpaf = a.af[mref];
    const bool isimputed = !a.common[mref];
    const int psite = a.segm[mref];
    const int nchunks = (a.ntgt + SS_CHUNK - 1) / SS_CHUNK;
    // row strides of one target (two haplotype rows); a producer warp's next
    // target is SS_PROD targets further
    const size_t sD = (size_t)2 * a.ldd, sA = (size_t)2 * a.lda;
    const size_t sB = (size_t)4 * a.ldb, sG = (size_t)4 * a.ldg;   // in 32-bit words
    double adsum = 0.0, ad2sum = 0.0;   // summing warp
    int ac1 = 0, nv = 0;                // producers: alleles counted, dosages added (AN)
    unsigned long long conflicts = 0;
    // --improveCalls statistics of the CTA: no change, het->het, hom->hom, het->hom, hom->het
    __shared__ unsigned long long s_icnt[5];
    __shared__ double s_itot[5];
    if (threadIdx.x < 5) {
        s_icnt[threadIdx.x] = 0;
        s_itot[threadIdx.x] = 0.0;
    }
    __syncthreads();
    for (int c = 0; c <= nchunks; c++) {
        if (wid < SS_PROD && c < nchunks) {
            float(*bs)[32] = tsum[c & 1];
            float(*bq)[32] = tsq[c & 1];
            const int ib = c * SS_CHUNK + wid;   // this warp's first target of the chunk
            const float *dp = a.dos + (size_t)ib * sD + s;
            const uint32_t *bp = reinterpret_cast<const uint32_t *>(a.bits) + (size_t)ib * sB + (s >> 5);
            float *ap = a.ads + (size_t)ib * sA + s;
            uint32_t *gp32 = reinterpret_cast<uint32_t *>(a.gtbits) + (size_t)ib * sG + blockIdx.x;
            for (int k0 = 0; k0 < SS_PER; k0 += SS_U) {
                float r0[SS_U], r1[SS_U], q0[SS_U], q1[SS_U];
                uint32_t w0[SS_U], w1[SS_U], p01[SS_U];
                uint8_t g[SS_U];
#pragma unroll
                for (int u = 0; u < SS_U; u++) {
                    const int i = ib + (k0 + u) * SS_PROD;
                    if (i < a.ntgt) {
                        const float *d = dp + (size_t)(k0 + u) * SS_PROD * sD;
                        const uint32_t *b = bp + (size_t)(k0 + u) * SS_PROD * sB;
                        r0[u] = d[0];
                        r1[u] = d[a.ldd];
                        w0[u] = b[0];
                        w1[u] = b[2 * a.ldb];
                        if (!isimputed) {   // the typed site's call: genotype, phased alleles and dosages
                            g[u] = a.gt[(size_t)i * a.M + psite];
                            p01[u] = bit_at(a.phased + (size_t)(2 * i) * a.wM, psite) |
                                     bit_at(a.phased + (size_t)(2 * i + 1) * a.wM, psite) << 1;
                            q0[u] = a.pdos_mat[(size_t)i * a.ldp + psite];
                            q1[u] = a.pdos_pat[(size_t)i * a.ldp + psite];
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < SS_U; u++) {
                    const int k = k0 + u;
                    const int i = ib + k * SS_PROD;
                    if (i >= a.ntgt) break;   // uniform across the warp
                    int hap0, hap1;
                    float ads0, ads1;
                    if (HAP && a.haptgt[i]) {
                        // haploid target (:3192-3226 imputed, :3399-3437 typed): row 2i
                        // only; the second ADS and GP2 are "vector end".  A typed,
                        // non-missing call without --overwriteCalls keeps the phased
                        // allele with a missing ADS and adds nothing to AF, r2, AC or
                        // AN; the reference leaves DS and GP unset there (its worker
                        // buffers keep an earlier site's values): written here as DS
                        // missing and GP (missing, end, end)
                        float term = 0.0f, sq = 0.0f, dsv, g0f, g1f;
                        if (isimputed || a.overwriteCalls || g[u] == 3) {
                            hap0 = (w0[u] >> (s & 31)) & 1u;
                            ads0 = r0[u];
                            if (ads0 < 0.0f) { ads0 = rpaf; hap0 = rpaf > 0.5f; conflicts++; }
                            term = ads0;
                            sq = __fmul_rn(ads0, ads0);
                            nv++;
                            ac1 += hap0;
                            dsv = ads0;
                            g0f = one_minus(ads0);
                            g1f = ads0;
                        } else {
                            hap0 = p01[u] & 1u;
                            ads0 = bcf_missing();
                            dsv = bcf_missing();
                            g0f = bcf_missing();
                            g1f = bcf_vector_end();
                        }
                        hap1 = 0;
                        bs[k * SS_PROD + wid][lane] = term;
                        bq[k * SS_PROD + wid][lane] = sq;
                        if (valid) {
                            float *o = ap + (size_t)k * SS_PROD * sA;
                            o[0] = ads0;
                            o[a.lda] = bcf_vector_end();
                            if (DS) a.ds[(size_t)i * a.lda + s] = dsv;
                            if (GP) {
                                float *gp = a.gp + (size_t)i * 3 * a.lda;
                                gp[s] = g0f;
                                gp[a.lda + s] = g1f;
                                gp[2 * (size_t)a.lda + s] = bcf_vector_end();
                            }
                        }
                    } else {
                        if (isimputed || a.overwriteCalls || g[u] == 3) {   // :3126-3152, :3246-3270
                            hap0 = (w0[u] >> (s & 31)) & 1u;
                            hap1 = (w1[u] >> (s & 31)) & 1u;
                            ads0 = r0[u];
                            ads1 = r1[u];
                            if (ads0 < 0.0f) { ads0 = rpaf; hap0 = rpaf > 0.5f; conflicts++; }
                            if (ads1 < 0.0f) { ads1 = rpaf; hap1 = rpaf > 0.5f; conflicts++; }
                        } else {   // :3272-3340: the phased call
                            hap0 = p01[u] & 1u;
                            hap1 = p01[u] >> 1;
                            ads0 = q0[u];
                            ads1 = q1[u];
                            if (a.improveCalls) {
                                const float i0raw = r0[u], i1raw = r1[u];
                                float idos0 = i0raw < 0.0f ? rpaf : i0raw;
                                float idos1 = i1raw < 0.0f ? rpaf : i1raw;
                                if (idos0 > 0.5f) idos0 = one_minus(idos0);
                                if (idos1 > 0.5f) idos1 = one_minus(idos1);
                                const float pdos0 = ads0 > 0.5f ? one_minus(ads0) : ads0;
                                const float pdos1 = ads1 > 0.5f ? one_minus(ads1) : ads1;
                                const float improve0 = __fsub_rn(pdos0, idos0), improve1 = __fsub_rn(pdos1, idos1);
                                const float improve = __fadd_rn(improve0, improve1);
                                if (improve > 0.0f) {
                                    conflicts += (i0raw < 0.0f) + (i1raw < 0.0f);
                                    const int n0 = (w0[u] >> (s & 31)) & 1u, n1 = (w1[u] >> (s & 31)) & 1u;
                                    // :3306-3330: which alleles the imputed call changes
                                    const bool c0 = hap0 != n0, c1 = hap1 != n1, het = hap0 != hap1;
                                    const int cat = (c0 && c1) ? (het ? 1 : 2) : (c0 || c1) ? (het ? 3 : 4) : 0;
                                    if (valid && a.icnt) {
                                        atomicAdd(&s_icnt[cat], 1ull);
                                        atomicAdd(&s_itot[cat], (double)improve);
                                    }
                                    hap0 = n0;
                                    hap1 = n1;
                                    ads0 = hap0 ? one_minus(idos0) : idos0;
                                    ads1 = hap1 ? one_minus(idos1) : idos1;
                                }
                            }
                        }
                        // :3154-3175, :3342-3361 -- the float terms of the double sums
                        bs[k * SS_PROD + wid][lane] = __fadd_rn(ads0, ads1);
                        bq[k * SS_PROD + wid][lane] = __fadd_rn(__fmul_rn(ads0, ads0), __fmul_rn(ads1, ads1));
                        if (valid) {
                            float *o = ap + (size_t)k * SS_PROD * sA;
                            o[0] = ads0;
                            o[a.lda] = ads1;
                            if (DS) a.ds[(size_t)i * a.lda + s] = __fadd_rn(ads0, ads1);
                            if (GP) {
                                const double g0 = __dmul_rn(__dsub_rn(1.0, (double)ads0), __dsub_rn(1.0, (double)ads1));
                                const double g2 = (double)__fmul_rn(ads0, ads1);
                                const double g1 = __dsub_rn(__dsub_rn(1.0, g0), g2);
                                float *gp = a.gp + (size_t)i * 3 * a.lda;
                                gp[s] = (float)g0;
                                gp[a.lda + s] = (float)g1;
                                gp[2 * (size_t)a.lda + s] = (float)g2;
                            }
                        }
                        ac1 += hap0 + hap1;
                        nv += 2;
                    }
                    // the written alleles as bits: the warp's 32 sites are one 32-bit word of each row
                    const unsigned b0 = __ballot_sync(0xffffffffu, valid && hap0);
                    const unsigned b1 = __ballot_sync(0xffffffffu, valid && hap1);
                    if (lane == 0) {
                        uint32_t *gw = gp32 + (size_t)k * SS_PROD * sG;
                        gw[0] = b0;
                        gw[2 * a.ldg] = b1;
                    }
                }
            }
        } else if (wid == SS_PROD && c > 0) {   // the previous chunk's terms, in target order
            const int pc = c - 1;
            const int nt = min(SS_CHUNK, a.ntgt - pc * SS_CHUNK);
            float(*bs)[32] = tsum[pc & 1];
            float(*bq)[32] = tsq[pc & 1];
            for (int t = 0; t < nt; t++) {
                adsum = __dadd_rn(adsum, (double)bs[t][lane]);
                ad2sum = __dadd_rn(ad2sum, (double)bq[t][lane]);
            }
        }
        __syncthreads();
    }
    if (wid < SS_PROD) {
        wac[wid][lane] = ac1;
        wnv[wid][lane] = nv;
        if (!valid) conflicts = 0;   // lanes past the last site computed site 0's values
        for (int o = 16; o; o >>= 1) conflicts += __shfl_xor_sync(0xffffffffu, conflicts, o);
        if (lane == 0 && conflicts) atomicAdd(a.conflicts, conflicts);
    }
    __syncthreads();
    if (a.icnt && threadIdx.x < 5 && s_icnt[threadIdx.x]) {
        atomicAdd(a.icnt + threadIdx.x, s_icnt[threadIdx.x]);
        atomicAdd(a.itot + threadIdx.x, s_itot[threadIdx.x]);
    }
    if (wid != SS_PROD || !valid) return;
    int nval = 0;   // dosages added: two per diploid target, one or none per haploid one
    for (int w = 0; w < SS_PROD; w++) {
        ac1 += wac[w][lane];
        nval += wnv[w][lane];
    }
    // :3363-3383, minimac4's r2
    double r2 = 1.0, af = 0.0;
    if (nval) {
        af = __ddiv_rn(adsum, (double)nval);
        const double evar = __dmul_rn(af, __dsub_rn(1.0, af));
        const double ovar = __ddiv_rn(__dsub_rn(ad2sum, __dmul_rn(adsum, af)), (double)nval);
        r2 = (evar > 0.0 && ovar > 0.0) ? __ddiv_rn(ovar, evar) : 0.0;
    }
    const float r2f = (float)r2, aff = (float)af;
    const float maff = aff > 0.5f ? __fsub_rn(1.0f, aff) : aff;
    a.r2[isite] = r2f;
    a.af_out[isite] = aff;
    a.maf[isite] = maff;
    a.ac[isite] = ac1;
    a.an[isite] = nval;   // AN counts the alleles whose dosages were added
    a.pass[isite] = !(r2f < a.r2filter || maff < a.maffilter);
}

template <bool HAP>
void launch_site_stats_t(const SiteStatsArgs &a, dim3 grid, dim3 block, cudaStream_t st) {
    if (a.ds && a.gp) site_stats_kernel<true, true, HAP><<<grid, block, 0, st>>>(a);
    else if (a.ds) site_stats_kernel<true, false, HAP><<<grid, block, 0, st>>>(a);
    else if (a.gp) site_stats_kernel<false, true, HAP><<<grid, block, 0, st>>>(a);
    else site_stats_kernel<false, false, HAP><<<grid, block, 0, st>>>(a);
}

cudaError_t launch_site_stats(const SiteStatsArgs &a, cudaStream_t st) {
    if (a.nsites <= 0) return cudaSuccess;
    const dim3 grid((a.nsites + 31) / 32), block((SS_PROD + 1) * 32);
    // haploid targets in a separate instantiation: the diploid one keeps its registers
    if (a.haptgt) launch_site_stats_t<true>(a, grid, block, st);
    else launch_site_stats_t<false>(a, grid, block, st);
    return cudaGetLastError();
}

}  // namespace eimp
