// Per-site output statistics of an imputed bunch (sm_100a).
//
//  site_stats_kernel -- the numeric part of VCFData::writeVCFImputedBunch
//                       (VCFData.cpp:3068-3446) for diploid targets: the
//                       allele dosage and allele written for every target
//                       haplotype (imputation conflicts take the reference
//                       panel's allele frequency, typed sites keep the phased
//                       call unless --overwriteCalls / --improveCalls), the
//                       optional DS and GP fields, and per site AC, AN, the
//                       dosage AF and MAF, the minimac4 r2 and whether the
//                       record passes the r2 / MAF output filters.
//
// One thread per reference site walks the targets in order, so the double
// sums that feed AF and r2 are accumulated in the reference's order and with
// its roundings (float sums of a target's two dosages, added into doubles).
// For a fixed target the threads of a warp read 32 consecutive dosages of the
// haplotype's row: every load and store is coalesced.  HBM-bound: each site
// reads the 2N dosages and writes the 2N allele dosages.
#include "common.cuh"
#include "kernels.h"

namespace eimp {

constexpr int SS_U = 8;   // targets whose inputs a thread loads ahead

__device__ __forceinline__ float one_minus(float x) {   // `1.0 - x` with x float, rounded back to float
    return (float)__dsub_rn(1.0, (double)x);
}

__global__ void __launch_bounds__(128) site_stats_kernel(SiteStatsArgs a) {
    const int isite = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = isite < a.nsites;
    const int s = valid ? isite : 0;
    const int mref = a.mref_begin + s;
    const float rpaf = a.af[mref];
    const bool isimputed = !a.common[mref];
    const int psite = a.segm[mref];
    double adsum = 0.0, ad2sum = 0.0;
    int nval = 0, ac1 = 0, an = 0;
    unsigned long long conflicts = 0;
    // targets in batches of SS_U: the batch's dosages and allele words are
    // loaded first (SS_U loads of each row in flight per thread), then the
    // targets are processed in order
    for (int i0 = 0; i0 < a.ntgt; i0 += SS_U) {
        float r0[SS_U], r1[SS_U], q0[SS_U], q1[SS_U];
        uint32_t w0[SS_U], w1[SS_U], p01[SS_U];
        uint8_t g[SS_U];
#pragma unroll
        for (int u = 0; u < SS_U; u++) {
            const int i = i0 + u;
            if (i < a.ntgt) {
                r0[u] = a.dos[(size_t)(2 * i) * a.ldd + s];
                r1[u] = a.dos[(size_t)(2 * i + 1) * a.ldd + s];
                w0[u] = reinterpret_cast<const uint32_t *>(a.bits + (size_t)(2 * i) * a.ldb)[s >> 5];
                w1[u] = reinterpret_cast<const uint32_t *>(a.bits + (size_t)(2 * i + 1) * a.ldb)[s >> 5];
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
            const int i = i0 + u;
            if (i >= a.ntgt) break;   // uniform across the warp
            const int h0 = 2 * i, h1 = 2 * i + 1;
            int hap0, hap1;
            float ads0, ads1;
            const bool use_imp = isimputed || a.overwriteCalls || g[u] == 3;
            if (use_imp) {   // :3126-3152, :3246-3270
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
                    if (__fadd_rn(improve0, improve1) > 0.0f) {
                        conflicts += (i0raw < 0.0f) + (i1raw < 0.0f);
                        hap0 = (w0[u] >> (s & 31)) & 1u;
                        hap1 = (w1[u] >> (s & 31)) & 1u;
                        ads0 = hap0 ? one_minus(idos0) : idos0;
                        ads1 = hap1 ? one_minus(idos1) : idos1;
                    }
                }
            }
            // :3154-3175, :3342-3361
            adsum = __dadd_rn(adsum, (double)__fadd_rn(ads0, ads1));
            ad2sum = __dadd_rn(ad2sum, (double)__fadd_rn(__fmul_rn(ads0, ads0), __fmul_rn(ads1, ads1)));
            if (valid) {
                a.ads[(size_t)h0 * a.lda + s] = ads0;
                a.ads[(size_t)h1 * a.lda + s] = ads1;
                if (a.ds) a.ds[(size_t)i * a.lda + s] = __fadd_rn(ads0, ads1);
                if (a.gp) {
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
            an += 2;
            nval += 2;
            // the written alleles as bits: the warp's 32 sites are one 32-bit word of each row
            const unsigned b0 = __ballot_sync(0xffffffffu, valid && hap0);
            const unsigned b1 = __ballot_sync(0xffffffffu, valid && hap1);
            if (lane == 0 && isite - lane < a.nsites) {
                reinterpret_cast<uint32_t *>(a.gtbits + (size_t)h0 * a.ldg)[isite >> 5] = b0;
                reinterpret_cast<uint32_t *>(a.gtbits + (size_t)h1 * a.ldg)[isite >> 5] = b1;
            }
        }
    }
    if (!valid) return;
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
    a.an[isite] = an;
    a.pass[isite] = !(r2f < a.r2filter || maff < a.maffilter);
    if (conflicts) atomicAdd(a.conflicts, conflicts);
}

cudaError_t launch_site_stats(const SiteStatsArgs &a, cudaStream_t st) {
    if (a.nsites <= 0) return cudaSuccess;
    site_stats_kernel<<<(a.nsites + 127) / 128, 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace eimp
