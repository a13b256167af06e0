/*
 * eimp_gpu.h -- C ABI of the B200 (sm_100a) implementation of EagleImp's
 * data-parallel hot path: condensed-reference build, PBWT + beam phasing and
 * PBWT imputation.
 *
 * Conventions (same as the reference):
 *  - bit vectors are uint64 words, least significant bit first, each row padded
 *    to whole 512-bit units: W(n) = ceil(n/512)*8 words (Datatypes.h:70);
 *  - genotypes are one byte per site: 0 hom-ref, 1 het, 2 hom-alt, 3 missing
 *    (Datatypes.h:81-86);
 *  - all functions return 0 on success and a non-zero EIMP_E_* code otherwise;
 *    eimp_last_error() then describes the failure (the reference throws
 *    thrust::system_error from checkCUDAError, GPUKernels.h:29-38, or calls
 *    StatusFile::addError + exit; callers map a non-zero return to that);
 *  - a context is bound to one CUDA device and one stream; calls on one context
 *    must not overlap (one context per host thread, as the reference keeps one
 *    GPUEngine per preprocessing thread, PBWTPhaser.cpp:484-488).
 * There is no CPU fallback: every entry point runs CUDA kernels and fails when
 * no device is present.
 */
#ifndef EIMP_GPU_H_
#define EIMP_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    EIMP_OK = 0,
    EIMP_E_CUDA = 1,        /* a CUDA runtime call failed */
    EIMP_E_ARG = 2,         /* invalid argument or call order */
    EIMP_E_CAPACITY = 3,    /* a fixed-capacity device structure overflowed */
    EIMP_E_BEAM_EMPTY = 4,  /* "Beam is empty. No paths left." (Beam.cpp:466-470) */
    EIMP_E_NOMEM = 5        /* device allocation failed */
};

typedef struct eimp_ctx eimp_ctx;

/* Phasing parameters; defaults of the reference in brackets (Args.cpp:274-299,
 * main.cpp:207-237, 305-306, 326).
 * Limits of this implementation, each returning EIMP_E_ARG when exceeded (the
 * reference accepts any size_t): K after clamping at most 65,536; hsize,
 * hsize_fast and the history lengths hsize*hist at most 128 (BooleanHistory
 * keeps 128 sites); beamwidth and beamwidth_fast at most 128 (the beam
 * kernel's per-warp arrays); the reference's defaults are inside all of them.
 * A phasing reference whose typed sites need more than the device's opt-in
 * shared memory per block for two genotype bit vectors (16 x W(M) bytes;
 * 929,792 sites on a B200) returns EIMP_E_CAPACITY. */
typedef struct {
    int K;              /* conditioning haplotypes [10000], clamped to Nrefhaps */
    int hsize;          /* history size H [100] */
    int beamwidth;      /* beam width P [128] */
    int delta;          /* call delay Delta [24] */
    int hsize_fast;     /* pre-phasing history [30] */
    int beamwidth_fast; /* pre-phasing beam width [64] */
    int delta_fast;     /* pre-phasing delta [10] */
    float cMmaxsplit;   /* [0.125] */
    float expectIBDcM;  /* [2.0] */
    float hist;         /* history factor [1.0] */
    float pErr;         /* genotype error probability [0.003] */
    float pLimit;       /* beam probability limit [= pErr] */
    float minfixsize, maxfixsize, minfixthr, maxfixthr;   /* [0.5, 0.9, 0.99, 1.0] */
    int doPrePhasing;   /* [0] */
    int doRevPhasing;   /* [1] */
} eimp_phase_params;

/* ---------------------------------------------------------------- context */

/* Opens a context on CUDA device `device` (replaces GPUEngine::GPUEngine(int),
 * GPUEngine.h:45). */
int eimp_create(int device, eimp_ctx **out);
/* Frees all device memory of the context (GPUEngine::free, GPUEngine.h:64). */
void eimp_destroy(eimp_ctx *ctx);
/* Human-readable description of the last failure on this context. */
const char *eimp_last_error(const eimp_ctx *ctx);
/* Blocks until all work on the context's stream is done; returns
 * EIMP_E_CAPACITY / EIMP_E_BEAM_EMPTY if a kernel launched since the last
 * check reported one (the *_dev entry points do not synchronise). */
int eimp_synchronize(eimp_ctx *ctx);
/* Number of kernels this context has launched so far. */
uint64_t eimp_kernel_launches(const eimp_ctx *ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that order their own
 * work with it. */
void *eimp_stream(eimp_ctx *ctx);

/* Device timing of the phasing stages (no counterpart in the reference; a
 * diagnostic).  With timing on, every eimp_phase_targets* call records CUDA
 * events on the context's stream around its stages; eimp_phase_stage_ms then
 * waits for the last call and writes up to n of its stage times in ms: best
 * haplotypes + call sites, the host read of the split counts, the condensed
 * reference, the PBWTs, the beam. */
int eimp_set_timing(eimp_ctx *ctx, int on);
int eimp_phase_stage_ms(eimp_ctx *ctx, float *ms, int n);

/* CUDA-graph form of a batch step (no counterpart in the reference; the
 * reference launches per block from host threads).  eimp_capture_begin starts
 * capturing the context's stream; the *_dev entry points called next are
 * recorded instead of run (their work on the context's second stream joins
 * the capture through the events that order it); eimp_capture_end
 * instantiates the graph, and eimp_graph_launch replays it on the context's
 * stream with the same buffers.  Phasing must run in capacity mode
 * (eimp_phase_reserve) to be captured: in the default mode it reads the
 * split counts back to the host to size the condensed reference. */
int eimp_capture_begin(eimp_ctx *ctx);
int eimp_capture_end(eimp_ctx *ctx);
int eimp_graph_launch(eimp_ctx *ctx);

/* ------------------------------------------ GPUEngine drop-in (cref + PBWT) */

/* GPUEngine::initialize (GPUEngine.h:50, GPUEngine.cu:44-96): uploads the typed
 * reference in site-major layout (M rows of refTCapacity bytes, haplotype bits
 * of NrefhapsAD haplotypes).  Kwords = W(K). */
int eimp_gpu_initialize(eimp_ctx *ctx, size_t K, size_t Kwords, size_t M, size_t Nrefhapscorr,
                        size_t NrefhapsAD, size_t refTCapacity, const uint64_t *refTData);
/* GPUEngine::getBlockSize (GPUEngine.h:53): targets per runCrefPBWT call. */
size_t eimp_gpu_block_size(const eimp_ctx *ctx);
/* GPUEngine::runCrefPBWTKernel (GPUEngine.h:55-61, GPUEngine.cu:98-217) for
 * ntgt <= block size targets.  Per target t: tgtData[t] = GenotypeVector data
 * (interleaved is0/is2 words), splitData[t] = split-site flags (W(M) words),
 * besthapData[t] = best-haplotype flags (W(NrefhapsAD) words);
 * crefTOffsets = exclusive prefix of (2*S_t+1), ntgt+1 entries.  Output:
 * cPBWT[t] = forward rows then backward rows (sweep order), 4*Kwords uint32
 * per row ([data, cumulative zeros] pairs, 1-padded tail word, zero padding
 * words); count0s[t] = zeros per condensed row (2*S_t+1 ints). */
int eimp_gpu_run_cref_pbwt(eimp_ctx *ctx, size_t ntgt, const uint64_t *const *tgtData,
                           const uint64_t *const *splitData, const uint64_t *const *besthapData,
                           const uint32_t *crefTOffsets, uint32_t *const *cPBWT, int *const *count0s);

/* ------------------------------------------------------------- phasing */

/* Uploads the typed reference for phasing: hapmajor (nhaps x W(M) words,
 * VCFData::reference, VCFData.h:199), sitemajor (M x W(nhaps) words,
 * VCFData::referenceT, VCFData.h:201) and the genetic positions of the typed
 * sites in cM (VCFData::cMs, VCFData.h:227). */
int eimp_phase_set_reference(eimp_ctx *ctx, size_t M, size_t nhaps, const uint64_t *hapmajor,
                             const uint64_t *sitemajor, const float *cM);

/* The same from a panel already in device memory (no counterpart in the
 * reference, whose VCFData builds reference/referenceT while reading): the
 * rows d_typed[0..M-1] of the site-major panel d_sitemajor_full (rows of
 * ldw_words >= W(nhaps) words) are the typed sites; their haplotype-major
 * transpose is built on the device.  d_cM: M genetic positions.  Enqueued on
 * the context's stream; the device buffers must stay valid until it ran. */
int eimp_phase_set_reference_dev(eimp_ctx *ctx, size_t M, size_t nhaps, const uint64_t *d_sitemajor_full,
                                 size_t ldw_words, const int64_t *d_typed, const float *d_cM);

/* Target::prepPhase (Target.cpp:95-163) for a batch of targets, on the device:
 * best haplotypes (K ascending indices per target), best-haplotype flags
 * (W(nhaps) words), monomorphic sites (W(M) words), split sites and call
 * locations (capacity M each, counts in nsplits / ncalls) and the split-site cM
 * differences (capacity M+1).  gt: ntgt x M genotype bytes.  Any output pointer
 * may be NULL. */
int eimp_phase_prep(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *gt,
                    int32_t *besthaps, uint64_t *flags, uint64_t *monos, int32_t *splits, int32_t *calls,
                    float *cmdiffs, int32_t *nsplits, int32_t *ncalls);

/* Target::condensedReferenceT + PBWT construction (Target.cpp:250-282,
 * PBWT.cpp:33-70) for a batch: returns in *rows_out the total number of
 * condensed rows sum_t (2*S_t+1); with cref/count0/pbwt non-NULL also copies
 * the condensed reference (rows x W(K) words), count0 (rows) and the
 * compressed PBWT (2*rows x 2*ceil(K/32) uint32: per target the forward rows
 * then the backward rows in sweep order) -- call once with NULL buffers to size
 * them. */
int eimp_phase_cref_pbwt(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *gt,
                         size_t *rows_out, int64_t *rowoff, uint64_t *cref, int32_t *count0, uint32_t *pbwt);

/* Target::phase (Target.cpp:166-289) for a batch of diploid targets: mats/pats
 * ntgt x W(M) words, dos_mats/dos_pats ntgt x M floats, totalconf and
 * ncallsites per target (Target.h:73-74). */
/* Phasing iterations after the first (PBWTPhaser.cpp:406-476): the phasing
 * reference is the panel followed by the phased targets of the previous
 * iteration (target t as sample first_sample + t), and target t of the
 * following phasing calls leaves its own sample out of its best haplotypes
 * (Target::findBestHaps, Target.cpp:791-811), K at most the panel's
 * haplotypes minus 2.  first_sample < 0 turns it off (the first iteration).
 * No counterpart function in the reference, which passes the index through
 * its Target objects. */
int eimp_phase_exclude_self(eimp_ctx *ctx, int64_t first_sample);

/* Chunked runs (VCFData.cpp:2802-2816, Target.cpp:311-312, 443): the maternal
 * phase of every target's first heterozygous site, carried over from the
 * overlap with the previous chunk (0 = Ref, 1 = Alt; VCFData::getStartPhase),
 * for the next phasing calls, which must then phase exactly ntgt targets.
 * ntgt = 0 goes back to Ref for all (the first chunk). */
int eimp_phase_start_phases(eimp_ctx *ctx, size_t ntgt, const uint8_t *phases);

/* Haploid samples of the phasing reference (chrX males and other haploid
 * regions; VCFData::getHaploidsRef, read with the Qref, VCFData.cpp:2157-2209):
 * nsamples = Nrefhaps/2 flags, 1 = haploid.  A haploid sample's second
 * haplotype column is a placeholder (a homozygous copy) that no target
 * chooses (Target.cpp:800-806, 830-838), and K is clamped to the haplotypes
 * that exist: Nrefhaps less one per haploid sample, less the target's own two
 * in iterations after the first (PBWTPhaser.cpp:159, 210).  In iterations
 * after the first the flags cover the reference followed by the phased
 * targets, haploid targets flagged as the reference does (VCFData.cpp:1926-1931).
 * Call after eimp_phase_set_reference, which resets all samples to diploid;
 * haploid = NULL (or no flag set) means all diploid. */
int eimp_phase_set_haploid_ref(eimp_ctx *ctx, size_t nsamples, const uint8_t *haploid);

/* Haploid targets of the next phasing calls (VCFData::getHaploidsTgt): ntgt
 * flags, 1 = haploid; the calls must then phase exactly ntgt targets.  A
 * haploid target is not phased (Target.cpp:166-203): its genotypes (0, 2, 3 =
 * missing) become the maternal haplotype and dosage, missing sites stay Ref
 * with dosage 0 (the reference's default without --impMissing), the
 * confidence and the number of call sites are its non-missing sites, and its
 * paternal haplotype and dosages are zero.  A heterozygous genotype in a
 * haploid target returns EIMP_E_ARG ("Found heterozygous genotype in haploid
 * target.").  ntgt = 0 goes back to all diploid. */
int eimp_phase_haploid_targets(eimp_ctx *ctx, size_t ntgt, const uint8_t *haploid);

/* Launch shapes (no counterpart in the reference; the results do not depend
 * on them), per context, for the autotuner (eimp_b200/autotune.py):
 *   EIMP_SHAPE_DOSAGE_SPAN     64-site tiles per warp of the dosage kernel: 4, 8 [default] or 16
 *   EIMP_SHAPE_SMM_WARPS       warps (target haplotypes) per CTA of the match search: 1, 2 [default] or 4
 *   EIMP_SHAPE_BEAM_SLOTS_PCT  warps of the persistent beam launch, in % of the warps that can be
 *                              resident at once: 1..100 [default 100]
 *   EIMP_SHAPE_SMM_TREE_POOLS  1 [default]: a match tree that could outgrow its shared-memory pool
 *                              moves to a global-memory pool and its warp goes on; 0: such a
 *                              haplotype is redone from its first site by the retry launch
 * A value outside these returns EIMP_E_ARG and changes nothing. */
enum { EIMP_SHAPE_DOSAGE_SPAN = 0, EIMP_SHAPE_SMM_WARPS = 1, EIMP_SHAPE_BEAM_SLOTS_PCT = 2,
       EIMP_SHAPE_SMM_TREE_POOLS = 3 };
int eimp_set_launch_shape(eimp_ctx *ctx, int knob, int value);
int eimp_get_launch_shape(const eimp_ctx *ctx, int knob, int *value);

/* Capacity mode for phasing (no counterpart in the reference): reserves the
 * batch buffers for up to max_targets targets and max_rows condensed rows
 * (sum over the targets of 2*S_t+1).  Afterwards the row offsets are computed
 * on the device, so a phasing call makes no host round trip and can be
 * captured; a batch that needs more rows skips the condensed reference, the
 * PBWT and the beam and reports EIMP_E_CAPACITY at the next status check.
 * max_rows = 0 returns to the default mode. */
int eimp_phase_reserve(eimp_ctx *ctx, const eimp_phase_params *p, size_t max_targets, size_t max_rows);

int eimp_phase_targets(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *gt,
                       uint64_t *mats, uint64_t *pats, float *dos_mats, float *dos_pats, float *totalconf,
                       int32_t *ncallsites);

/* ----------------------------------------------------------- imputation */

/* Reference for PBWTImputer (PBWTImputer.cpp:31-185): the full reference in
 * site-major layout (Mref x W(nhaps) words, VCFData::referenceFullT,
 * VCFData.h:211), its allele frequencies (Mref floats), the typed sites (M
 * ascending indices into the full reference, VCFData::indexToRefFull) and the
 * typed reference in site-major layout (M x W(nhaps) words).  Builds the
 * reference PBWT with its prefix arrays on the device.  The build runs on a
 * second stream of the context, after the work already queued on the main
 * stream and concurrently with what is queued there next (e.g. the phasing of
 * the same batch); the calls that read the reference wait for it. */
int eimp_imp_set_reference(eimp_ctx *ctx, size_t Mref, size_t nhaps, const uint64_t *sitemajor_full,
                           const float *af_full, size_t M, const int64_t *typed, const uint64_t *sitemajor_typed);

/* PBWTImputer::prepareImputation (PBWTImputer.cpp:63-185): set-maximal matches
 * of ntargets diploid targets.  phased: 2*ntargets x W(M) words (mat, pat per
 * target, as phasedTargets); gt: ntargets x M genotype bytes (missing = 3,
 * VCFData::tgtmiss).  match_cap = matches stored per haplotype (0: M/4+64). */
int eimp_imp_prepare(eimp_ctx *ctx, size_t ntargets, const uint64_t *phased, const uint8_t *gt,
                     int setmaxerrors, int imputeCalls, size_t match_cap);

/* Haploid samples of the imputation reference (PBWTImputer.cpp:31-34,
 * 67-114): nsamples = nhaps/2 flags, 1 = haploid.  The reference PBWT and
 * its prefix arrays then hold K = nhaps - (haploid samples) haplotypes, the
 * first column of every sample and the second of the diploid ones, and the
 * dosages read the panel through that column map (VCFData::getHaploidsRefMap,
 * TargetImp.cpp:536).  Applies to the next eimp_imp_set_reference[_dev],
 * which must then have nhaps = 2 * nsamples; NULL = all diploid. */
int eimp_imp_set_haploid_ref(eimp_ctx *ctx, size_t nsamples, const uint8_t *haploid);

/* Haploid targets of the next eimp_imp_prepare[_dev] (ntgt must equal its
 * ntargets): only the first haplotype of a haploid target is searched and
 * imputed (PBWTImputer.cpp:31, 130, 202); its second row of matches is empty
 * and its second row of dosages and alleles is zero in eimp_imp_bunch and
 * left unwritten by eimp_imp_bunch_dev.  The output statistics do not support
 * haploid targets (EIMP_E_ARG).  ntgt = 0 or NULL: all diploid. */
int eimp_imp_haploid_targets(eimp_ctx *ctx, size_t ntgt, const uint8_t *haploid);

/* PBWTImputer::imputeBunch (PBWTImputer.cpp:187-204) for the window of nsites
 * reference sites starting at mref_begin: bits 2*ntargets x W(nsites) words,
 * dos 2*ntargets x nsites floats.  Sites the reference imputes get the
 * imputed allele and dosage (uncovered sites: dosage -1, DOSAGE_CONFLICT,
 * TargetImp.cpp:26); typed non-missing sites, which the reference leaves
 * unwritten, get the phased allele as bit and 0.0/1.0 dosage. */
int eimp_imp_bunch(eimp_ctx *ctx, size_t mref_begin, size_t nsites, uint64_t *bits, float *dos);

/* Set-maximal matches found for one target haplotype: returns their number in
 * *n; with out non-NULL copies up to cap matches as int32 quadruples (start,
 * end, refstart, refend) -- TargetImp::Match, TargetImp.h:64-75. */
int eimp_imp_matches(eimp_ctx *ctx, size_t hap, int32_t *out, size_t cap, size_t *n);

/* Reference PBWT of the imputer: compressed rows (M x 2*ceil(nhaps/32) uint32)
 * and prefix arrays ((M+1) x nhaps int32, PBWT::getSortOrder, PBWT.h:67). */
int eimp_imp_refpbwt(eimp_ctx *ctx, uint32_t *compr, int32_t *absperm);

/* gAbsPerm[site][lo..hi] (PBWT.h:67) of the reference PBWT, to the host
 * (site <= M: the order before typed site 'site').  For checking dosages
 * against an oracle on a sample without copying all (M+1) x K prefix
 * entries. */
int eimp_imp_prefix_slice(eimp_ctx *ctx, size_t site, size_t lo, size_t hi, int32_t *out);

/* Bit-matrix transpose on the device (no counterpart in the reference, whose
 * VCFData builds referenceT and reference while reading): d_src has 'rows'
 * rows of src_ld 64-bit words holding 'cols' bits each (LSB first); row c of
 * d_dst (stride dst_ld words) gets bit c of every source row, the first
 * ceil(rows/64) words written.  cols <= 65535 * 64.  Enqueued on the
 * context's stream. */
int eimp_transpose_bits_dev(eimp_ctx *ctx, const uint64_t *d_src, size_t rows, size_t src_ld, uint64_t *d_dst,
                            size_t cols, size_t dst_ld);

/* Output statistics of an imputed bunch: the numeric part of
 * VCFData::writeVCFImputedBunch (VCFData.cpp:3068-3446), which main.cpp:454
 * calls after PBWTImputer::imputeBunch for every bunch.
 * Per target haplotype and site: the allele dosage written (ADS; an imputation
 * conflict takes the reference panel allele frequency RefPanelAF and the
 * allele RefPanelAF > 0.5; a typed, non-missing call keeps the phased allele
 * and dosage unless overwriteCalls, or improveCalls and the imputed dosage is
 * closer to 0/1), and the allele written (GT).  Optional per target and site:
 * DS = ADS0 + ADS1 and GP (three floats, VCFData.cpp:3159-3166).  Per site:
 * AF and MAF from the dosages, minimac4's r2, AC, AN and whether the record
 * passes the --imputeR2filter / --imputeMAFfilter thresholds.  `conflicts`
 * receives the number of conflicts (VCFData::conflictcnt).
 * Haploid targets (eimp_imp_haploid_targets; VCFData.cpp:3192-3226,
 * 3399-3437) use their first haplotype row: its ADS and allele, the second
 * row's ADS set to htslib's "vector end" (0x7F800002) and its GT bit 0, DS =
 * ADS0 and GP = (1 - ADS0, ADS0, vector end).  At a typed, non-missing site
 * (without overwriteCalls) a haploid target keeps its phased allele with ADS
 * "missing" (0x7F800001) and adds nothing to AF, r2, AC or AN; the reference
 * leaves DS and GP unset there (its writer buffers keep an earlier site's
 * values), and they are written as DS missing and GP (missing, vector end,
 * vector end).  The --improveCalls run statistics go to the context's
 * counters (eimp_imp_improve_stats). */
typedef struct {
    int overwriteCalls;   /* --overwriteCalls (Args.cpp:304) */
    int improveCalls;     /* --improveCalls (Args.cpp:305) */
    float r2filter;       /* --imputeR2filter (Args.cpp:283), default 0 */
    float maffilter;      /* --imputeMAFfilter (Args.cpp:284), default 0 */
} eimp_site_stats_opts;

/* Phased dosages of the prepared targets (phasedDosages of main.cpp: the mat
 * and pat dosage of each target at the typed sites, ntargets x M floats each,
 * as eimp_phase_targets returns them), kept on the device for the output
 * statistics; a new eimp_imp_prepare drops them. */
int eimp_imp_phased_dosages(eimp_ctx *ctx, const float *dos_mat, const float *dos_pat);

/* imputeBunch + the output statistics for the window [mref_begin,
 * mref_begin + nsites): ads 2*ntargets x nsites floats, gtbits 2*ntargets x
 * W(nsites) words, ds (NULL: skipped) ntargets x nsites, gp (NULL: skipped)
 * 3*ntargets x nsites floats (rows GP0, GP1, GP2 of each target), per site r2,
 * af, maf, ac, an, pass (nsites each), *conflicts. */
int eimp_imp_bunch_stats(eimp_ctx *ctx, size_t mref_begin, size_t nsites, const eimp_site_stats_opts *opts,
                         float *ads, uint64_t *gtbits, float *ds, float *gp, float *r2, float *af, float *maf,
                         int32_t *ac, int32_t *an, uint8_t *pass, uint64_t *conflicts);

/* The --improveCalls run statistics (VCFData's improvecnt* and totalimprove*
 * members, VCFData.cpp:3306-3330, reported in the run summary): improved calls
 * counted over every output-statistics call of the context with improveCalls
 * set, since the context was made or last reset.  counts[5] and totals[5] (the
 * sums of the calls' improvements) in the order: no allele change, het->het,
 * hom->hom, het->hom, hom->het.  reset != 0 zeroes them after the read.
 * Synchronises the context's stream.  The counts are exact; the device adds
 * the totals in an order of its own, so their last bits can differ from a
 * sequential sum (the reference's own order depends on its thread count). */
int eimp_imp_improve_stats(eimp_ctx *ctx, uint64_t *counts, double *totals, int reset);

/* Qref reference panel, haplotype section (qref_spec.md section I; read by
 * VCFData::qRefLoadNextVariant, VCFData.cpp:2378-2535, with runlengthDecode,
 * utils.h:194-): Mref variants, each <encsize uint64> followed by encsize
 * run-length bytes, or by the raw vector of W(2*Nref) words when encsize is
 * 0.  Decoded into Mref rows of W(2*Nref) words (bit 2s mat, 2s+1 pat of
 * sample s; the site-major referenceFullT layout, VCFData.h:211).  Masked
 * reference samples (--excludeRefSamples): eimp_qref_decode_masked below.
 *
 * eimp_qref_index (host only, no device): the byte offset of every variant's
 * <encsize> field; EIMP_E_ARG when the section is shorter than its variants
 * ("Failed reading haplotypes from reference.").
 * eimp_qref_decode: the section from host memory (copied once), decoded into
 * d_out (device, Mref rows of ldw_words words) or, when d_out is NULL, into a
 * buffer of the context; with host_out non-NULL the rows are also copied
 * there (Mref x W(2*Nref) words).  Returns EIMP_E_ARG for a truncated
 * run-length sequence ("Truncated runlength sequence!", utils.h:222-240). */
int eimp_qref_index(const uint8_t *section, size_t nbytes, size_t Mref, size_t Nref, int64_t *offsets);
int eimp_qref_decode(eimp_ctx *ctx, const uint8_t *section, size_t nbytes, size_t Mref, size_t Nref,
                     uint64_t *d_out, size_t ldw_words, uint64_t *host_out);
/* The same with masked reference samples (--excludeRefSamples;
 * VCFData::qRefLoadNextVariant VCFData.cpp:2378-2535, runlengthDecode
 * utils.h:194-): Nref samples in the section, masked[0..nmasked-1] ascending
 * sample indices to leave out (masked_haploid: 1 for a haploid sample),
 * nhaploid_ref haploid samples in the section.  Rows hold the
 * Nref - nmasked kept samples (W(2*(Nref-nmasked)) words); af (Mref floats,
 * the panel allele frequencies of the variants) is corrected in place for
 * the masked variant alleles as the reference does.  A raw vector and a
 * run-length code count a masked haploid sample stored as 01 or 10
 * differently, as the reference's two paths do. */
int eimp_qref_decode_masked(eimp_ctx *ctx, const uint8_t *section, size_t nbytes, size_t Mref, size_t Nref,
                            size_t nmasked, const int64_t *masked, const uint8_t *masked_haploid,
                            size_t nhaploid_ref, float *af, uint64_t *d_out, size_t ldw_words, uint64_t *host_out);

/* ------------------------------------------- device-resident variants ----
 * Same operations on device pointers (inputs already in HBM; outputs written to
 * device memory; no host<->device copies, no synchronisation). */
int eimp_imp_prepare_dev(eimp_ctx *ctx, size_t ntargets, const uint64_t *d_phased, const uint8_t *d_gt,
                         int setmaxerrors, int imputeCalls, size_t match_cap);
int eimp_imp_bunch_dev(eimp_ctx *ctx, size_t mref_begin, size_t nsites, uint64_t *d_bits, size_t ldb_words,
                       float *d_dos, size_t ldd);
/* d_sitemajor_typed may be NULL: the typed rows are then gathered from
 * d_sitemajor_full at d_typed on the device. */
int eimp_imp_set_reference_dev(eimp_ctx *ctx, size_t Mref, size_t nhaps, const uint64_t *d_sitemajor_full,
                               const float *d_af_full, size_t M, const int64_t *d_typed,
                               const uint64_t *d_sitemajor_typed);
/* The output statistics of a bunch already imputed into d_bits / d_dos
 * (eimp_imp_bunch_dev); phased dosages from d_pdos_mat / d_pdos_pat (ntargets
 * rows of ldp floats) or, when those are NULL, from eimp_imp_phased_dosages.
 * d_ads / d_gtbits may be d_dos / d_bits (in place, with lda == ldd); the
 * statistics add to *d_conflicts. */
int eimp_imp_site_stats_dev(eimp_ctx *ctx, size_t mref_begin, size_t nsites, const uint64_t *d_bits,
                            size_t ldb_words, const float *d_dos, size_t ldd, const float *d_pdos_mat,
                            const float *d_pdos_pat, size_t ldp, const eimp_site_stats_opts *opts, float *d_ads,
                            size_t lda, uint64_t *d_gtbits, size_t ldg_words, float *d_ds, float *d_gp,
                            float *d_r2, float *d_af, float *d_maf, int32_t *d_ac, int32_t *d_an, uint8_t *d_pass,
                            uint64_t *d_conflicts);
/* The Qref haplotype section already in device memory (readable up to the
 * next multiple of 4 bytes past its end) with its variant offsets from
 * eimp_qref_index; only enqueues the decode: a truncated sequence is
 * reported by the next eimp_synchronize. */
int eimp_qref_decode_dev(eimp_ctx *ctx, const uint8_t *d_section, const int64_t *d_offsets, size_t Mref,
                         size_t Nref, uint64_t *d_out, size_t ldw_words);
int eimp_phase_targets_dev(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *d_gt,
                           uint64_t *d_mats, uint64_t *d_pats, float *d_dos_mats, float *d_dos_pats,
                           float *d_totalconf, int32_t *d_ncallsites);

/* ------------------------------------------------ allocation-free variant ----
 * No counterpart in the reference.  Best-haplotype selection (the Hamming
 * counts and K-smallest choice of Target::findBestHaps) for callers that cannot
 * let this library allocate device memory -- e.g. a host framework that owns
 * the device budget through its own pool, or a serving loop that allows no
 * allocation after start-up.  It needs no context and calls no
 * cudaMalloc/cudaFree: the per-haplotype error counts live in a fixed device
 * array of EIMP_BESTHAPS_NOALLOC_MAX uint32 (16 MiB), which every GPU that
 * loads the library holds until the process exits.
 *  - all pointers are device pointers on the current device; `stream` is a
 *    cudaStream_t (NULL: the default stream); the call only enqueues work;
 *  - inputs: d_gt ntgt x M genotype bytes, d_hapmajor nhaps x W(M) words;
 *    outputs: d_besthaps ntgt x min(K, nhaps) ascending indices, d_flags
 *    ntgt x W(nhaps) words -- the same values eimp_phase_prep returns;
 *  - ntgt x nhaps must not exceed EIMP_BESTHAPS_NOALLOC_MAX, otherwise the call
 *    returns EIMP_E_CAPACITY and does nothing (split the targets into batches);
 *  - a target's genotype bit vectors are staged in shared memory (16 x W(M)
 *    bytes per CTA): M above the device's opt-in shared memory per block
 *    (929,792 typed sites on a B200) returns EIMP_E_CAPACITY as well;
 *  - the first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) and keeps it; make that call before capturing a
 *    stream on that device, and do not reset the device (cudaDeviceReset)
 *    after it, which would leave the kept address stale;
 *  - all calls on a device share the array: calls that overlap on the GPU
 *    (different streams, unsynchronised) race and give wrong results. */
#define EIMP_BESTHAPS_NOALLOC_MAX (4u << 20)
int eimp_besthaps_noalloc(void *stream, size_t ntgt, size_t M, const uint8_t *d_gt, const uint64_t *d_hapmajor,
                          size_t nhaps, size_t K, int32_t *d_besthaps, uint64_t *d_flags);

#ifdef __cplusplus
}
#endif

#endif /* EIMP_GPU_H_ */
