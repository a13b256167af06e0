// Kernel launchers shared between the translation units of libeimp_b200.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

// set-maximal match search: warps (target haplotypes) per CTA of the wide
// and the compact kernel, and the per-warp match-tree node pools in shared
// memory of the first launch and of the retry launch (one warp per CTA)
#define SMM_WARPS 4
#define SMMC_WARPS 2
#define SMM_NODES 512
#define SMM_NODES_RETRY 4096
// beam phasing: warps (targets) per CTA
#define BEAM_WARPS 4

namespace eimp {

// Raises a kernel's dynamic shared-memory limit to at least `bytes`; never
// lowers it.  The limit is a property of the kernel, shared by every host
// thread: launchers that set it to exactly their own size could lower it
// between another thread's setting and its launch.
cudaError_t ensure_dynamic_smem(const void *kernel, size_t bytes);


// ---- imputation (imp_kernels.cu)
// global scratch launch_refpbwt needs (0: none) for K haplotypes
size_t refpbwt_scratch_bytes(int K, int wN);
cudaError_t launch_refpbwt(const uint64_t *sitemajor, int M, int K, int wN, uint32_t *compr, int32_t *absperm,
                           int32_t *count0, int32_t *scratch, cudaStream_t st);
cudaError_t launch_transpose(const uint64_t *src, size_t rows, size_t srcw, uint64_t *dst, size_t cols, size_t dstw,
                             cudaStream_t st);
// the same with separate row strides; dstw words of each dst row are written
cudaError_t launch_transpose_ld(const uint64_t *src, size_t rows, size_t src_ld, uint64_t *dst, size_t cols,
                                size_t dstw, size_t dst_ld, cudaStream_t st);
// dst row i (w words) = src row idx[i] (rows ldsrc words apart)
cudaError_t launch_gather_rows(const uint64_t *src, size_t ldsrc, const int64_t *idx, int n, int w, uint64_t *dst,
                               cudaStream_t st);
// hapmap (null: identity): the target haplotype (row of phased, matches,
// outputs; its target = row / 2) of each of the nhaps haplotypes searched
// gpool: gpool_slots global tree pools of smm_gpool_slot_bytes(K) bytes for
// the compact kernel's trees that outgrow shared memory, handed out through
// *gpool_next (zero before the launch); NULL: none (such trees are retried)
cudaError_t launch_smm(const uint32_t *compr, const int32_t *count0, int M, int K, const uint64_t *phased, int wM,
                       const uint8_t *gt, int nhaps, const int32_t *hapmap, int setmaxerrors, int4 *matches, int cap,
                       int *nmatch, uint32_t *status, int warps, void *gpool, int gpool_slots, int *gpool_next,
                       cudaStream_t st);
size_t smm_gpool_slot_bytes(int K);
// refmap (null: identity): panel haplotype of each PBWT haplotype (the
// reduced reference without the haploid samples' placeholder columns)
cudaError_t launch_dosage(const int4 *matches, int cap, const int *nmatch, const int32_t *absperm, int K,
                          const int32_t *refmap, const uint64_t *hapmajor_full, int wMref, const int2 *sinfo,
                          const uint64_t *phased, int wM, const uint8_t *gt, int M, int nhaps, const int32_t *hapmap,
                          int mref_begin, int nsites, int imputeCalls, float *dos, int ldd, uint64_t *bits, int ldb,
                          int span, cudaStream_t st);
// segment map of the typed sites over the reference sites, plus the dosage
// kernel's per-site pair (segment | typed << 31, shortcut height | af>0.5 << 31)
cudaError_t launch_segmap(const int64_t *typed, int M, int Mref, const float *af, int nrefhaps_total, int32_t *segm,
                          uint8_t *common, int2 *sinfo, cudaStream_t st);

// ---- output statistics of an imputed bunch (site_stats.cu)
struct SiteStatsArgs {
    int ntgt, mref_begin, nsites;
    const uint64_t *bits; int ldb;            // imputed alleles, 2*ntgt rows of ldb words
    const float *dos; int ldd;                // imputed dosages, 2*ntgt rows (-1: conflict)
    const uint64_t *phased; int wM;           // phased haplotypes at the typed sites
    const float *pdos_mat, *pdos_pat; int ldp;   // phased dosages, ntgt rows each
    const uint8_t *gt; int M;                 // target genotypes at the typed sites (3: missing)
    const int32_t *segm; const uint8_t *common; const float *af;   // per reference site
    int overwriteCalls, improveCalls;
    float r2filter, maffilter;
    float *ads; int lda;                      // allele dosages written, 2*ntgt rows
    uint64_t *gtbits; int ldg;                // alleles written, 2*ntgt rows of ldg words
    float *ds, *gp;                           // optional: ntgt rows / 3*ntgt rows of lda floats
    float *r2, *af_out, *maf;                 // per site of the bunch
    int32_t *ac, *an;
    uint8_t *pass;
    unsigned long long *conflicts;            // incremented by the conflicts found
    const uint8_t *haptgt;                    // per target, 1 = haploid (NULL: all diploid)
    unsigned long long *icnt;                 // --improveCalls run statistics, added to:
    double *itot;                             //   5 counts and 5 totals (NULL: not kept)
};
cudaError_t launch_site_stats(const SiteStatsArgs &a, cudaStream_t st);

// ---- Qref haplotype section (qref_decode.cu)
cudaError_t launch_qref_decode(const uint8_t *sec, const int64_t *offs, int Mref, int nwords, uint64_t *out,
                               size_t ldw, uint32_t *status, cudaStream_t st);
cudaError_t launch_qref_mask(const uint8_t *sec, const int64_t *offs, int nvar, const uint64_t *rows, size_t ldr,
                             const int32_t *kept, int nkept, int nwout, const int64_t *masked, int nmasked,
                             const uint8_t *masked_hap, float an_before, float an_after, float *af, uint64_t *out,
                             size_t ldo, cudaStream_t st);

// ---- phasing preparation, condensed reference, PBWT (phase_prep.cu)
// haploid: per reference sample, 1 = haploid (its second column is never
// chosen); null: all diploid
cudaError_t launch_besthaps(const uint8_t *gt, int ntgt, int M, const uint64_t *hapmajor, int nhaps, int wM, int K,
                            uint32_t *nerr_scratch, int32_t *besthaps, uint64_t *flags, int wN, int self0,
                            const uint8_t *haploid, cudaStream_t st);
// tgt_haploid: per target, 1 = haploid (no split sites); null: all diploid
cudaError_t launch_monos_calls(const uint8_t *gt, int ntgt, int M, const uint64_t *hapmajor, int wM,
                               const int32_t *besthaps, int K, const float *cm, float cMmaxsplit, uint64_t *monos,
                               int32_t *splits, int32_t *calls, float *cmdiffs, int32_t *nsplits, int32_t *ncalls,
                               const uint8_t *tgt_haploid, cudaStream_t st);
// outputs of the haploid targets of a batch (written after the beam)
cudaError_t launch_haploid_phase(const uint8_t *gt, int ntgt, int M, int wM, const uint8_t *tgt_haploid,
                                 uint64_t *mats, uint64_t *pats, float *dmat, float *dpat, float *totalconf,
                                 int32_t *ncallsites, uint32_t *status, cudaStream_t st);
// dst row r bit j = src row r bit map[j], j < ncols; a second haplotype (odd
// map value) at a word's first column is zero, as the reference's
// setPairWithPreInit leaves it
cudaError_t launch_compact_cols(const uint64_t *src, int rows, int srcw, const int32_t *map, int ncols, uint64_t *dst,
                                int dstw, cudaStream_t st);
// condensed reference from the haplotype-major reference (nhaps x wM words)
cudaError_t launch_cref(const uint8_t *gt, int ntgt, int M, const uint64_t *hapmajor, int wM, int nhaps,
                        const int32_t *besthaps, int K, const int32_t *splits, const int32_t *nsplits,
                        const int64_t *rowoff, uint64_t *cref, const int *skip, cudaStream_t st);
// forward and backward PBWT of the condensed references; writes count0 too
cudaError_t launch_pbwt(const uint64_t *cref, int32_t *count0, const int64_t *rowoff, int ntgt, int K,
                        uint32_t *pbwt, size_t rowstride, int emit_padded, const int *skip, cudaStream_t st);
// row offsets of the condensed references on the device (exclusive prefix of
// 2*nsplits+1); sets *skip (and the status flag) when they exceed cap rows
cudaError_t launch_rowoff(const int32_t *nsplits, int ntgt, int64_t *rowoff, int64_t cap, int *skip,
                          uint32_t *status, cudaStream_t st);

// ---- beam phasing (beam.cu)
struct BeamParams {
    int K;
    int H, P, Delta;      // history length (hsize*hist rounded), beam width, call delay
    int Hf, Pf, Deltaf;   // the same for the pre-phasing beam
    float expectIBDcM, pErr, pLimit;
    float minfixsize, maxfixsize, minfixthr, maxfixthr;
    int doPrePhasing, doRevPhasing;
    // maternal phase of each target's first heterozygous site, carried over
    // from the previous chunk (VCFData::getStartPhase; 0 = Ref); null: all Ref
    const uint8_t *startph = nullptr;
};
size_t beam_arena_bytes(const BeamParams &p, int S_max);
// warps of the persistent beam launch for ntgt targets (a multiple of the
// warps per CTA; at most the resident ones), -1 on a CUDA error
int beam_slots(const BeamParams &p, int M, int ntgt, int pct = 100);
// the persistent beam: slots warps (beam_slots), one arena of arena_bytes per
// slot; order (ntgt ints) and workq (one int) are scratch: the longest-first
// order and the queue counter, both filled here
cudaError_t launch_beam(const BeamParams &p, int ntgt, int M, const uint8_t *gt, const uint64_t *monos,
                        const int32_t *splits, const int32_t *nsplits, const int32_t *calls, const int32_t *ncalls,
                        const float *cmdiffs, const uint32_t *pbwt, const int32_t *count0, const int64_t *rowoff,
                        void *arena, size_t arena_bytes, int slots, int32_t *order, int *workq, uint64_t *mats,
                        uint64_t *pats, float *dmat, float *dpat, float *totalconf, int32_t *ncallsites,
                        uint32_t *status, const int *skip, cudaStream_t st);

}  // namespace eimp
