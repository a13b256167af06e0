/*
 * CPU restatement of EagleImp's data-parallel hot path -- TEST ORACLE.
 *
 * This is test infrastructure: only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it, as the checker.  The product (the
 * CUDA library in eimp_b200/) never calls it.  Every function follows the
 * reference file:line named beside it; the restatement is pinned against the
 * reference's own sources compiled by oracle/Makefile (target "ref") and
 * against the golden fixtures under tests/golden/.
 *
 * Layouts (all bit vectors are uint64 words, LSB first, rows padded to
 * 512-bit units, W(n) = ceil(n/512)*8 words -- Datatypes.h:70):
 *   gt          genotype codes 0/1/2, 3 = missing, one byte per typed site
 *   hapmajor    typed reference, one row of W(M) words per haplotype
 *   sitemajor   typed reference, one row of W(N) words per typed site
 *   cref        condensed reference, (2S+1) rows of W(K) words
 *   pbwt rows   2*ceil(K/32) uint32 per row: [data, cumulative zeros] pairs
 */
#ifndef EIMP_ORACLE_H_
#define EIMP_ORACLE_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

size_t eo_W(size_t nbits);

/* a1+a2: Target::findBestHaps (Target.cpp:779-875) with the Hamming count of
 * GenotypeVector::compare_withPreInit (Datatypes.cpp:107-116).
 * gtw: interleaved is0/is2 words (2*W(M)); nerr_out (optional, nhaps). */
void eo_besthaps(const uint64_t *gtw, const uint64_t *hapmajor, size_t nhaps, size_t wM,
                 size_t K, int64_t *besthaps, uint32_t *nerr_out);

/* a3: Target::findMonos (Target.cpp:878-897) -> monos (wM words) */
void eo_monos(const uint64_t *hapmajor, size_t wM, size_t M, const int64_t *besthaps, size_t K,
              uint64_t *monos);

/* a3: Target::findCallLocs (Target.cpp:900-950).  Returns S (number of
 * split sites); fills splits[S], calls[*ncalls], cmdiffs[S+1] (when S>0). */
long eo_calllocs(const uint8_t *gt, const uint64_t *monos, const float *cm, size_t M,
                 float cMmaxsplit, int64_t *splits, int64_t *calls, size_t *ncalls, float *cmdiffs);

/* a4: Target::condensedReferenceT (Target.cpp:953-1038) -> cref rows (2S+1)
 * x W(K) words (cleared here), count0[2S+1]. */
void eo_cref(const uint8_t *gt, const uint64_t *sitemajor, size_t M, size_t nhaps,
             const int64_t *besthaps, size_t K, const int64_t *splits, size_t S,
             uint64_t *cref, int32_t *count0);

/* a5: PBWT::buildComprPBWT (PBWT.cpp:207-285) over Mp rows of K bits (row
 * stride rowwords words).  reverse: sweep rows Mp-1..0, output in sweep
 * order.  out: Mp x 2*ceil(K/32) uint32.  absperm (optional, forward only):
 * (Mp+1) x K prefix arrays.  count0_out (optional): zeros per input row. */
void eo_pbwt(const uint64_t *rows, size_t rowwords, size_t Mp, size_t K, int reverse,
             uint32_t *out, int32_t *absperm, int32_t *count0_out);

/* a6: PBWT::decodeRelPerm (PBWT.cpp:367-382) */
int eo_rank(const uint32_t *row, int cnt0, int from);

/* a8: TargetImp::calcSMMatches (TargetImp.cpp:74-246) for one target
 * haplotype.  hap: W(M) words; miss: sorted missing positions.  Returns the
 * number of matches written to out (4 int64 per match: start, end,
 * refstart, refend) or -1 if more than maxmatches. */
long eo_smmatches(const uint32_t *refpbwt, const int32_t *count0, size_t M, size_t K,
                  const uint64_t *hap, const int64_t *miss, size_t nmiss, int setmaxerrors,
                  int64_t *out, size_t maxmatches);

/* largest number of live match-tree nodes seen by eo_smmatches in this process */
int eo_smm_peak_nodes(void);

/* a9: TargetImp::imputeBunch (TargetImp.cpp:474-558) over all Mref sites of
 * one target haplotype, block 0, no forwarding.  bits: W(Mref) words
 * (cleared here); dos: Mref floats; imputed (optional): 1 where the
 * reference writes a dosage.  Where it writes none (typed, non-missing
 * sites without imputeCalls) the phased allele of hap (W(M) words) is
 * written as bit and 0.0/1.0 dosage. */
void eo_impute(const int64_t *matches, size_t nmatches, const int32_t *absperm, size_t K,
               const uint64_t *sitemajor_full, size_t wN, size_t Mref, const int64_t *typed,
               size_t M, const float *af_full, size_t nrefhaps_total, const int64_t *miss,
               size_t nmiss, int imputeCalls, const uint64_t *hap, uint64_t *bits, float *dos,
               uint8_t *imputed, double *dos64);

/* Output statistics of an imputed bunch: the numeric part of
 * VCFData::writeVCFImputedBunch (VCFData.cpp:3068-3446).
 * Site-major over the bunch's nsites sites (site s = reference site
 * mref_begin + s):
 *   bits   2*ntgt rows of wb words (imputed alleles), dos 2*ntgt x nsites
 *   phased 2*ntgt rows of wM words, pdm/pdp ntgt x M phased dosages
 *   gt     ntgt x M genotype codes (3 = missing), typed_idx / is_typed per
 *          reference site (the typed index of the last typed site <= mref)
 *   haploid ntgt flags or NULL (haploid targets: row 2i only)
 * Outputs: ads 2*ntgt x nsites, gtbits 2*ntgt rows of wb words (zeroed by the
 * caller), ds ntgt x nsites (optional), gp 3*ntgt x nsites (optional, rows
 * GP0, GP1, GP2 per target), per site r2, af, maf, ac, an, pass; the
 * --improveCalls run statistics are added to improve_counts[5] and
 * improve_totals[5] (optional; VCFData.cpp:3306-3330); returns the number of
 * imputation conflicts.  Pinned to the reference's own writer
 * (oracle/_ref/libeimp_refwriter.so) by tests/test_site_stats_reference_writer.py. */
/* Qref haplotype vectors (qref_spec.md section I).
 * eo_rle_encode: runlengthEncode + addRunlength (utils.h:133-191) of nwords
 * words; returns the encoded length, or -1 where the reference gives up (the
 * encoding would not be shorter than the source).  enc needs nwords*8+3 bytes.
 * eo_rle_decode: runlengthDecode (utils.h:194-) without masked samples into
 * nwords zeroed words; returns 0, or -1 for a truncated sequence.
 * eo_qref_decode: the section of Mref variants (<encsize u64> then encsize
 * bytes, or the raw capacity bytes when encsize is 0 -- VCFData.cpp:2378-2535)
 * into Mref rows of nwords words; returns 0, -1 for a truncated sequence, -2
 * for a section shorter than its variants. */
long eo_rle_encode(const uint64_t *src, size_t nwords, uint8_t *enc);
int eo_rle_decode(const uint8_t *enc, size_t encsize, uint64_t *dest, size_t nwords);
int eo_qref_decode(const uint8_t *section, size_t nbytes, size_t Mref, size_t nwords, uint64_t *out);

long eo_site_stats(size_t ntgt, size_t mref_begin, size_t nsites, const uint64_t *bits, size_t wb,
                   const float *dos, const uint64_t *phased, size_t wM, const float *pdm, const float *pdp,
                   const uint8_t *gt, size_t M, const int32_t *typed_idx, const uint8_t *is_typed,
                   const float *af_full, const uint8_t *haploid, int overwriteCalls, int improveCalls,
                   float r2filter, float maffilter, float *ads, uint64_t *gtbits, float *ds, float *gp, float *r2,
                   float *af, float *maf, int32_t *ac, int32_t *an, uint8_t *pass, uint64_t *improve_counts,
                   double *improve_totals);

/* a7: phasing parameters (Args.cpp:274-299 defaults) */
typedef struct {
    int K;
    int hsize, beamwidth, delta;
    int hsize_fast, beamwidth_fast, delta_fast;
    float cMmaxsplit, expectIBDcM, hist, pErr, pLimit;
    float minfixsize, maxfixsize, minfixthr, maxfixthr;
    int doPrePhasing, doRevPhasing;
} eo_phase_params;

/* a7: Target::phase (Target.cpp:166-289) -> phaseExtPBWT (Target.cpp:291-777)
 * for one diploid target.  mat/pat: W(M) words (cleared here); dos_*: M
 * floats.  Returns 0, or a negative error code (-1 "beam is empty"). */
int eo_phase(const uint8_t *gt, const uint64_t *hapmajor, const uint64_t *sitemajor,
             const float *cm, size_t M, size_t nhaps, const eo_phase_params *p,
             uint64_t *mat, uint64_t *pat, float *dos_mat, float *dos_pat,
             float *totalconf, size_t *ncallsites);

/* phase targets [0, n) in parallel (OpenMP, dynamic 1) */
int eo_phase_many(const uint8_t *gt, size_t n, const uint64_t *hapmajor, const uint64_t *sitemajor,
                  const float *cm, size_t M, size_t nhaps, const eo_phase_params *p, int nthreads,
                  uint64_t *mats, uint64_t *pats, float *dos_mats, float *dos_pats);

#ifdef __cplusplus
}
#endif

#endif
