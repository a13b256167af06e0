// C ABI of libeimp_b200 (include/eimp_gpu.h): context, device buffers, and the
// host-facing entry points that mirror the reference's GPUEngine,
// Target::prepPhase/phase and PBWTImputer interfaces.
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.h"
#include "../../include/eimp_gpu.h"

using namespace eimp;

namespace {

// grow-only device buffer
struct DBuf {
    void *p = nullptr;
    size_t n = 0;
    ~DBuf() { if (p) cudaFree(p); }
    cudaError_t reserve(size_t bytes) {
        if (bytes <= n) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; n = 0; }
        cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
        if (e == cudaSuccess) n = bytes;
        return e;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

}  // namespace

struct eimp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // the imputation reference (transposed panel, segment map, reference
    // PBWT) is built on a side stream, so that it overlaps whatever the main
    // stream runs next (the phasing of the same batch); ref_ready marks its
    // end and every use on the main stream waits for it
    cudaStream_t side = nullptr;
    cudaEvent_t ref_ready = nullptr, main_mark = nullptr;
    // optional device timing of the phasing stages (eimp_set_timing)
    bool timing = false, tvalid = false;
    cudaEvent_t tev[6] = {};
    // capacity mode (eimp_phase_reserve): row offsets computed on the device
    // against a reserved row capacity; cur_skip = the device flag the
    // phasing kernels check (null outside capacity mode)
    int64_t rows_cap = 0;
    DBuf skipbuf;
    const int *cur_skip = nullptr;
    // stream capture (eimp_capture_begin / _end) and the instantiated graph
    bool capturing = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::string err;
    uint64_t launches = 0;
    DBuf status;
    // launch shapes (eimp_set_launch_shape)
    int shape_dos_span = 8, shape_smm_warps = SMMC_WARPS, shape_beam_pct = 100, shape_smm_pools = 1;

    // GPUEngine drop-in
    size_t g_K = 0, g_Kwords = 0, g_M = 0, g_Ncorr = 0, g_NAD = 0, g_refTcap = 0;
    DBuf g_refT, g_hapT, g_gt, g_splits, g_nsplits, g_bh, g_rowoff, g_cref, g_count0, g_pbwt;

    // phasing reference
    size_t p_M = 0, p_nhaps = 0;
    // phasing iterations after the first: reference sample of target 0 (-1: none)
    int64_t self0 = -1;
    // start phases of the targets of the next phasing calls (chunk carry)
    DBuf startph;
    size_t startph_n = 0;
    // ploidy: haploid samples of the phasing reference (count, device flags)
    // and haploid targets of the next phasing calls
    size_t p_nhaploid = 0;
    DBuf p_haploid;
    DBuf tgthap;
    size_t tgthap_n = 0;
    DBuf p_hapmajor, p_sitemajor, p_cm;
    // phasing batch scratch
    DBuf b_gt, b_nerr, b_bh, b_flags, b_monos, b_splits, b_calls, b_cmd, b_nsplits, b_ncalls, b_rowoff, b_cref,
        b_count0, b_pbwt, b_arena, b_out_mat, b_out_pat, b_out_dm, b_out_dp, b_out_tc, b_out_nc, b_order,
        b_workq;
    size_t b_rows = 0;

    // imputation reference; with haploid panel samples the PBWT holds i_K <
    // i_nhaps haplotypes, i_refmap their panel columns, i_sitetyped_c the
    // typed rows reduced to them
    size_t i_Mref = 0, i_nhaps = 0, i_M = 0, i_K = 0;
    size_t i_refhap_samples = 0, i_refK = 0;
    DBuf i_refmap, i_sitetyped_c;
    // haploid targets of the imputation: i_hapmap = row of each existing
    // target haplotype (i_ntgthaps of them) for i_tgthap_n targets
    size_t i_tgthap_n = 0, i_ntgthaps = 0;
    DBuf i_hapmap, i_tgtflag;
    DBuf i_hapfull, i_sitefull_tmp, i_af, i_typed, i_segm, i_common, i_sinfo, i_sitetyped_tmp, i_compr,
        i_absperm, i_count0, i_rpscratch;
    // prepared targets
    size_t i_ntargets = 0;
    int i_imputeCalls = 0;
    size_t i_cap = 0;
    DBuf i_phased, i_gt, i_matches, i_nmatch;
    // global tree pools of the match search (trees that outgrow shared memory) and their counter
    DBuf i_gpool, i_gnext;
    // host <-> device staging for bunches
    DBuf i_bits, i_dos;
    // phased dosages (eimp_imp_phased_dosages) and staging of the output statistics
    DBuf i_pdm, i_pdp, s_ads, s_gt, s_ds, s_gp, s_site, s_conf;
    // --improveCalls run statistics: 5 counts then 5 double totals, added to
    // by every output-statistics call (VCFData's improvecnt*/totalimprove*)
    DBuf s_improve;
    // Qref haplotype section staging
    DBuf q_sec, q_offs, q_out, q_rows, q_mask, q_maskhap, q_kept, q_af;
    bool i_have_pdos = false;
};

namespace {

int fail(eimp_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? EIMP_E_NOMEM : EIMP_E_CUDA,         \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

#define LAUNCH(call)                                                                               \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        ctx->launches++;                                                                           \
        if (e_ != cudaSuccess) return fail(ctx, EIMP_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int use_device(eimp_ctx *ctx) {
    CK(cudaSetDevice(ctx->device));
    return 0;
}

// phasing stage boundaries: 0 start, 1 after prep, 2 before the condensed
// reference (after the host read of the split counts), 3 after it, 4 after
// the PBWT, 5 after the beam
void tmark(eimp_ctx *ctx, int i) {
    if (ctx->timing && !ctx->capturing) cudaEventRecord(ctx->tev[i], ctx->stream);
}

int check_status(eimp_ctx *ctx) {
    uint32_t st = 0;
    CK(cudaMemcpyAsync(&st, ctx->status.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (st) {
        CK(cudaMemsetAsync(ctx->status.p, 0, sizeof(uint32_t), ctx->stream));
        if (st & EIMP_ERR_BEAM_EMPTY) return fail(ctx, EIMP_E_BEAM_EMPTY, "Beam is empty. No paths left.");
        if (st & EIMP_ERR_QREF_TRUNCATED) return fail(ctx, EIMP_E_ARG, "Truncated runlength sequence!");
        if (st & EIMP_ERR_HAPLOID_HET) return fail(ctx, EIMP_E_ARG, "Found heterozygous genotype in haploid target.");
        char b[160];
        snprintf(b, sizeof b, "device structure capacity exceeded (status 0x%x)", st);
        return fail(ctx, EIMP_E_CAPACITY, b);
    }
    return 0;
}

// K of a phasing call: at most the haplotypes a target may choose from --
// all of the panel, or all but its own two in iterations after the first
// (PBWTPhaser.cpp:408-476: localK = min(K, localNrefhapsCorr))
size_t phase_K(const eimp_ctx *ctx, const eimp_phase_params *p) {
    // PBWTPhaser.cpp:159, 210: one haplotype less per haploid sample of the
    // panel, and the target's own two in iterations after the first
    size_t corr = ctx->p_nhaps - ctx->p_nhaploid;
    if (ctx->self0 >= 0) corr = corr >= 2 ? corr - 2 : 0;
    return (size_t)p->K < corr ? (size_t)p->K : corr;
}

}  // namespace

extern "C" {

int eimp_create(int device, eimp_ctx **out) {
    if (!out) return EIMP_E_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return EIMP_E_CUDA;
    if (device < 0 || device >= n) return EIMP_E_ARG;
    eimp_ctx *ctx = new eimp_ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ref_ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->main_mark, cudaEventDisableTiming) != cudaSuccess ||
        ctx->status.reserve(sizeof(uint32_t)) != cudaSuccess || cudaMemset(ctx->status.p, 0, sizeof(uint32_t)) != cudaSuccess ||
        ctx->s_improve.reserve(80) != cudaSuccess || cudaMemset(ctx->s_improve.p, 0, 80) != cudaSuccess) {
        if (ctx->main_mark) cudaEventDestroy(ctx->main_mark);
        if (ctx->ref_ready) cudaEventDestroy(ctx->ref_ready);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return EIMP_E_CUDA;
    }
    *out = ctx;
    return 0;
}

void eimp_destroy(eimp_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaStream_t s = ctx->stream, sd = ctx->side;
    cudaEvent_t e1 = ctx->ref_ready, e2 = ctx->main_mark;
    for (cudaEvent_t e : ctx->tev)
        if (e) cudaEventDestroy(e);
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    if (ctx->graph) cudaGraphDestroy(ctx->graph);
    delete ctx;
    if (e1) cudaEventDestroy(e1);
    if (e2) cudaEventDestroy(e2);
    if (sd) cudaStreamDestroy(sd);
    if (s) cudaStreamDestroy(s);
}

const char *eimp_last_error(const eimp_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int eimp_synchronize(eimp_ctx *ctx) {
    if (!ctx) return EIMP_E_ARG;
    CK(cudaStreamSynchronize(ctx->side));
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

uint64_t eimp_kernel_launches(const eimp_ctx *ctx) { return ctx ? ctx->launches : 0; }

int eimp_set_timing(eimp_ctx *ctx, int on) {
    if (!ctx) return EIMP_E_ARG;
    if (int r = use_device(ctx)) return r;
    if (on)
        for (cudaEvent_t &e : ctx->tev)
            if (!e) CK(cudaEventCreate(&e));
    ctx->timing = on != 0;
    ctx->tvalid = false;
    return 0;
}

int eimp_phase_stage_ms(eimp_ctx *ctx, float *ms, int n) {
    if (!ctx || !ms || n < 0) return EIMP_E_ARG;
    if (!ctx->tvalid) return fail(ctx, EIMP_E_ARG, "eimp_phase_stage_ms: timing off or no phasing call since it was set");
    if (int r = use_device(ctx)) return r;
    CK(cudaEventSynchronize(ctx->tev[5]));
    for (int i = 0; i < n && i < 5; i++) CK(cudaEventElapsedTime(&ms[i], ctx->tev[i], ctx->tev[i + 1]));
    return 0;
}

int eimp_capture_begin(eimp_ctx *ctx) {
    if (!ctx) return EIMP_E_ARG;
    if (ctx->capturing) return fail(ctx, EIMP_E_ARG, "eimp_capture_begin: already capturing");
    if (int r = use_device(ctx)) return r;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    ctx->capturing = true;
    return 0;
}

int eimp_capture_end(eimp_ctx *ctx) {
    if (!ctx) return EIMP_E_ARG;
    if (!ctx->capturing) return fail(ctx, EIMP_E_ARG, "eimp_capture_end: not capturing");
    if (int r = use_device(ctx)) return r;
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    ctx->capturing = false;
    CK(e);
    if (ctx->gexec) { cudaGraphExecDestroy(ctx->gexec); ctx->gexec = nullptr; }
    if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
    ctx->graph = g;
    CK(cudaGraphInstantiate(&ctx->gexec, g, 0));
    // events last recorded inside the capture belong to the graph; record
    // them again on their streams so that eager calls can wait on them
    CK(cudaEventRecord(ctx->ref_ready, ctx->side));
    CK(cudaEventRecord(ctx->main_mark, ctx->stream));
    return 0;
}

int eimp_graph_launch(eimp_ctx *ctx) {
    if (!ctx) return EIMP_E_ARG;
    if (!ctx->gexec) return fail(ctx, EIMP_E_ARG, "eimp_graph_launch: nothing captured");
    if (int r = use_device(ctx)) return r;
    CK(cudaGraphLaunch(ctx->gexec, ctx->stream));
    return 0;
}

void *eimp_stream(eimp_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int eimp_set_launch_shape(eimp_ctx *ctx, int knob, int value) {
    if (!ctx) return EIMP_E_ARG;
    switch (knob) {
    case EIMP_SHAPE_DOSAGE_SPAN:
        if (value != 4 && value != 8 && value != 16) return fail(ctx, EIMP_E_ARG, "dosage span: 4, 8 or 16 tiles");
        ctx->shape_dos_span = value;
        return 0;
    case EIMP_SHAPE_SMM_WARPS:
        if (value != 1 && value != 2 && value != 4) return fail(ctx, EIMP_E_ARG, "match-search warps per CTA: 1, 2 or 4");
        ctx->shape_smm_warps = value;
        return 0;
    case EIMP_SHAPE_BEAM_SLOTS_PCT:
        if (value < 1 || value > 100) return fail(ctx, EIMP_E_ARG, "beam slots: 1..100 % of the resident warps");
        ctx->shape_beam_pct = value;
        return 0;
    case EIMP_SHAPE_SMM_TREE_POOLS:
        if (value != 0 && value != 1) return fail(ctx, EIMP_E_ARG, "match-search tree pools: 0 or 1");
        ctx->shape_smm_pools = value;
        return 0;
    default:
        return fail(ctx, EIMP_E_ARG, "unknown launch-shape knob");
    }
}

int eimp_get_launch_shape(const eimp_ctx *ctx, int knob, int *value) {
    if (!ctx || !value) return EIMP_E_ARG;
    switch (knob) {
    case EIMP_SHAPE_DOSAGE_SPAN: *value = ctx->shape_dos_span; return 0;
    case EIMP_SHAPE_SMM_WARPS: *value = ctx->shape_smm_warps; return 0;
    case EIMP_SHAPE_BEAM_SLOTS_PCT: *value = ctx->shape_beam_pct; return 0;
    case EIMP_SHAPE_SMM_TREE_POOLS: *value = ctx->shape_smm_pools; return 0;
    default: return EIMP_E_ARG;
    }
}

// ------------------------------------------------------------------ imputation

int eimp_imp_set_reference_dev(eimp_ctx *ctx, size_t Mref, size_t nhaps, const uint64_t *d_sitemajor_full,
                               const float *d_af_full, size_t M, const int64_t *d_typed,
                               const uint64_t *d_sitemajor_typed) {
    if (!ctx || !Mref || !nhaps || !M || M > Mref) return fail(ctx, EIMP_E_ARG, "eimp_imp_set_reference: bad sizes");
    if (int r = use_device(ctx)) return r;
    // after everything already queued on the main stream (earlier batches
    // may still read the buffers rewritten here)
    CK(cudaEventRecord(ctx->main_mark, ctx->stream));
    CK(cudaStreamWaitEvent(ctx->side, ctx->main_mark, 0));
    cudaStream_t st = ctx->side;
    if (ctx->i_refhap_samples && 2 * ctx->i_refhap_samples != nhaps)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_set_reference: haploid flags were set for a different panel");
    // the PBWT's haplotypes: all, or without the haploid samples'
    // placeholder columns (PBWTImputer.cpp:31-34, 67-114)
    const size_t K = ctx->i_refhap_samples ? ctx->i_refK : nhaps;
    const size_t wN = eimp_W(nhaps), wMref = eimp_W(Mref), kw = eimp_kw(K);
    ctx->i_Mref = Mref; ctx->i_nhaps = nhaps; ctx->i_M = M; ctx->i_K = K;
    CK(ctx->i_hapfull.reserve(nhaps * wMref * 8));
    CK(ctx->i_af.reserve(Mref * 4));
    CK(ctx->i_typed.reserve(M * 8));
    CK(ctx->i_segm.reserve(Mref * 4));
    CK(ctx->i_common.reserve(Mref));
    CK(ctx->i_sinfo.reserve(Mref * sizeof(int2)));
    CK(ctx->i_compr.reserve(M * kw * 4));
    CK(ctx->i_absperm.reserve((M + 1) * K * 4));
    CK(ctx->i_count0.reserve(M * 4));
    CK(cudaMemcpyAsync(ctx->i_af.p, d_af_full, Mref * 4, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(ctx->i_typed.p, d_typed, M * 8, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemsetAsync(ctx->i_hapfull.p, 0, nhaps * wMref * 8, st));
    LAUNCH(launch_transpose(d_sitemajor_full, Mref, wN, ctx->i_hapfull.as<uint64_t>(), nhaps, wMref, st));
    LAUNCH(launch_segmap(ctx->i_typed.as<int64_t>(), (int)M, (int)Mref, ctx->i_af.as<float>(), (int)nhaps,
                         ctx->i_segm.as<int32_t>(), ctx->i_common.as<uint8_t>(), ctx->i_sinfo.as<int2>(), st));
    const uint64_t *typed_rows = d_sitemajor_typed;
    if (!typed_rows) {   // the typed sites' rows from the panel itself
        CK(ctx->i_sitetyped_tmp.reserve(M * wN * 8));
        LAUNCH(launch_gather_rows(d_sitemajor_full, wN, ctx->i_typed.as<int64_t>(), (int)M, (int)wN,
                                  ctx->i_sitetyped_tmp.as<uint64_t>(), st));
        typed_rows = ctx->i_sitetyped_tmp.as<uint64_t>();
    }
    size_t wK = wN;
    if (ctx->i_refhap_samples) {
        wK = eimp_W(K);
        CK(ctx->i_sitetyped_c.reserve(M * wK * 8));
        LAUNCH(launch_compact_cols(typed_rows, (int)M, (int)wN, ctx->i_refmap.as<int32_t>(), (int)K,
                                   ctx->i_sitetyped_c.as<uint64_t>(), (int)wK, st));
        typed_rows = ctx->i_sitetyped_c.as<uint64_t>();
    }
    const size_t rps = refpbwt_scratch_bytes((int)K, (int)wK);
    if (rps) CK(ctx->i_rpscratch.reserve(rps));
    LAUNCH(launch_refpbwt(typed_rows, (int)M, (int)K, (int)wK, ctx->i_compr.as<uint32_t>(),
                          ctx->i_absperm.as<int32_t>(), ctx->i_count0.as<int32_t>(),
                          rps ? ctx->i_rpscratch.as<int32_t>() : nullptr, st));
    CK(cudaEventRecord(ctx->ref_ready, st));
    return 0;
}

int eimp_imp_set_haploid_ref(eimp_ctx *ctx, size_t nsamples, const uint8_t *haploid) {
    if (!ctx) return EIMP_E_ARG;
    if (int r = use_device(ctx)) return r;
    size_t n = 0;
    for (size_t i = 0; haploid && i < nsamples; i++) n += haploid[i] != 0;
    if (!n) {   // all diploid: the PBWT over every column
        ctx->i_refhap_samples = 0;
        return 0;
    }
    // the existing haplotypes' panel columns, in panel order (VCFData.cpp:2191-2193)
    std::vector<int32_t> map;
    map.reserve(2 * nsamples - n);
    for (size_t i = 0; i < nsamples; i++) {
        map.push_back((int32_t)(2 * i));
        if (!haploid[i]) map.push_back((int32_t)(2 * i + 1));
    }
    CK(cudaStreamSynchronize(ctx->side));   // the map may be in use by a reference build
    CK(cudaStreamSynchronize(ctx->stream));
    CK(ctx->i_refmap.reserve(map.size() * 4));
    CK(cudaMemcpy(ctx->i_refmap.p, map.data(), map.size() * 4, cudaMemcpyHostToDevice));
    ctx->i_refhap_samples = nsamples;
    ctx->i_refK = map.size();
    return 0;
}

int eimp_imp_haploid_targets(eimp_ctx *ctx, size_t ntgt, const uint8_t *haploid) {
    if (!ctx) return EIMP_E_ARG;
    if (int r = use_device(ctx)) return r;
    size_t n = 0;
    for (size_t i = 0; haploid && i < ntgt; i++) n += haploid[i] != 0;
    if (!n) {
        ctx->i_tgthap_n = 0;
        return 0;
    }
    // the rows of the existing target haplotypes (VCFData.cpp:1340-1348)
    std::vector<int32_t> map;
    map.reserve(2 * ntgt - n);
    for (size_t i = 0; i < ntgt; i++) {
        map.push_back((int32_t)(2 * i));
        if (!haploid[i]) map.push_back((int32_t)(2 * i + 1));
    }
    CK(cudaStreamSynchronize(ctx->stream));   // the map may be in use by queued imputation work
    CK(ctx->i_hapmap.reserve(map.size() * 4));
    CK(cudaMemcpy(ctx->i_hapmap.p, map.data(), map.size() * 4, cudaMemcpyHostToDevice));
    // the flags themselves, for the output statistics (VCFData::haploidsTgt)
    std::vector<uint8_t> f(ntgt);
    for (size_t i = 0; i < ntgt; i++) f[i] = haploid[i] != 0;
    CK(ctx->i_tgtflag.reserve(ntgt));
    CK(cudaMemcpy(ctx->i_tgtflag.p, f.data(), ntgt, cudaMemcpyHostToDevice));
    ctx->i_tgthap_n = ntgt;
    ctx->i_ntgthaps = map.size();
    return 0;
}

int eimp_imp_set_reference(eimp_ctx *ctx, size_t Mref, size_t nhaps, const uint64_t *sitemajor_full,
                           const float *af_full, size_t M, const int64_t *typed, const uint64_t *sitemajor_typed) {
    if (!ctx || !sitemajor_full || !af_full || !typed || !sitemajor_typed)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_set_reference: NULL argument");
    if (int r = use_device(ctx)) return r;
    const size_t wN = eimp_W(nhaps);
    DBuf full, af, ty, st;
    CK(full.reserve(Mref * wN * 8));
    CK(af.reserve(Mref * 4));
    CK(ty.reserve(M * 8));
    CK(st.reserve(M * wN * 8));
    CK(cudaMemcpyAsync(full.p, sitemajor_full, Mref * wN * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(af.p, af_full, Mref * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ty.p, typed, M * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(st.p, sitemajor_typed, M * wN * 8, cudaMemcpyHostToDevice, ctx->stream));
    int r = eimp_imp_set_reference_dev(ctx, Mref, nhaps, full.as<uint64_t>(), af.as<float>(), M, ty.as<int64_t>(),
                                       st.as<uint64_t>());
    if (r) return r;
    CK(cudaStreamSynchronize(ctx->side));   // temporaries are freed on return
    return 0;
}

int eimp_imp_prepare_dev(eimp_ctx *ctx, size_t ntargets, const uint64_t *d_phased, const uint8_t *d_gt,
                         int setmaxerrors, int imputeCalls, size_t match_cap) {
    if (!ctx || !ctx->i_Mref) return fail(ctx, EIMP_E_ARG, "eimp_imp_prepare: no reference set");
    if (!ntargets) return fail(ctx, EIMP_E_ARG, "eimp_imp_prepare: no targets");
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->i_M, wM = eimp_W(M), nh = 2 * ntargets;
    size_t cap = match_cap ? match_cap : M / 4 + 64;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ref_ready, 0));
    ctx->i_ntargets = ntargets;
    ctx->i_have_pdos = false;   // phased dosages belong to the previous targets
    ctx->i_imputeCalls = imputeCalls;
    ctx->i_cap = cap;
    CK(ctx->i_phased.reserve(nh * wM * 8));
    CK(ctx->i_gt.reserve(ntargets * M));
    if (ctx->i_tgthap_n && ctx->i_tgthap_n != ntargets)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_prepare: haploid targets were set for a different number of targets");
    CK(ctx->i_matches.reserve(nh * cap * sizeof(int4)));
    CK(ctx->i_nmatch.reserve(nh * sizeof(int)));
    if (d_phased != ctx->i_phased.as<uint64_t>())
        CK(cudaMemcpyAsync(ctx->i_phased.p, d_phased, nh * wM * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    if (d_gt != ctx->i_gt.as<uint8_t>())
        CK(cudaMemcpyAsync(ctx->i_gt.p, d_gt, ntargets * M, cudaMemcpyDeviceToDevice, ctx->stream));
    // haploid targets: only their first haplotype is searched (PBWTImputer.cpp:31, 130)
    const int32_t *hapmap = ctx->i_tgthap_n ? ctx->i_hapmap.as<int32_t>() : nullptr;
    const size_t nsearch = ctx->i_tgthap_n ? ctx->i_ntgthaps : nh;
    if (hapmap) CK(cudaMemsetAsync(ctx->i_nmatch.p, 0, nh * sizeof(int), ctx->stream));
    // up to 2048 haplotypes per launch move a large tree to a global pool
    // instead of being redone by the retry launch
    const int gslots = ctx->shape_smm_pools ? (int)std::min<size_t>(nsearch, 2048) : 0;
    CK(ctx->i_gpool.reserve((size_t)gslots * smm_gpool_slot_bytes((int)ctx->i_K)));
    CK(ctx->i_gnext.reserve(sizeof(int)));
    CK(cudaMemsetAsync(ctx->i_gnext.p, 0, sizeof(int), ctx->stream));
    LAUNCH(launch_smm(ctx->i_compr.as<uint32_t>(), ctx->i_count0.as<int32_t>(), (int)M, (int)ctx->i_K,
                      ctx->i_phased.as<uint64_t>(), (int)wM, ctx->i_gt.as<uint8_t>(), (int)nsearch, hapmap,
                      setmaxerrors, ctx->i_matches.as<int4>(), (int)cap, ctx->i_nmatch.as<int>(),
                      ctx->status.as<uint32_t>(), ctx->shape_smm_warps, gslots ? ctx->i_gpool.p : nullptr, gslots,
                      ctx->i_gnext.as<int>(), ctx->stream));
    ctx->launches++;   // launch_smm launches twice: the small node pool, then the retry pass
    return 0;
}

int eimp_imp_prepare(eimp_ctx *ctx, size_t ntargets, const uint64_t *phased, const uint8_t *gt, int setmaxerrors,
                     int imputeCalls, size_t match_cap) {
    if (!ctx || !ctx->i_Mref) return fail(ctx, EIMP_E_ARG, "eimp_imp_prepare: no reference set");
    if (!phased || !gt) return fail(ctx, EIMP_E_ARG, "eimp_imp_prepare: NULL argument");
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->i_M, wM = eimp_W(M), nh = 2 * ntargets;
    CK(ctx->i_phased.reserve(nh * wM * 8));
    CK(ctx->i_gt.reserve(ntargets * M));
    CK(cudaMemcpyAsync(ctx->i_phased.p, phased, nh * wM * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->i_gt.p, gt, ntargets * M, cudaMemcpyHostToDevice, ctx->stream));
    int r = eimp_imp_prepare_dev(ctx, ntargets, ctx->i_phased.as<uint64_t>(), ctx->i_gt.as<uint8_t>(), setmaxerrors,
                                 imputeCalls, match_cap);
    if (r) return r;
    return check_status(ctx);
}

int eimp_imp_bunch_dev(eimp_ctx *ctx, size_t mref_begin, size_t nsites, uint64_t *d_bits, size_t ldb_words,
                       float *d_dos, size_t ldd) {
    if (!ctx || !ctx->i_ntargets) return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch: imputation not prepared");
    if (mref_begin + nsites > ctx->i_Mref || !nsites) return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch: window out of range");
    if (ldb_words < (nsites + 63) / 64 || ldd < nsites) return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch: leading dimension too small");
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->i_M;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ref_ready, 0));
    const int32_t *hapmap = ctx->i_tgthap_n ? ctx->i_hapmap.as<int32_t>() : nullptr;
    const size_t nimp = ctx->i_tgthap_n ? ctx->i_ntgthaps : 2 * ctx->i_ntargets;
    LAUNCH(launch_dosage(ctx->i_matches.as<int4>(), (int)ctx->i_cap, ctx->i_nmatch.as<int>(),
                         ctx->i_absperm.as<int32_t>(), (int)ctx->i_K,
                         ctx->i_refhap_samples ? ctx->i_refmap.as<int32_t>() : nullptr, ctx->i_hapfull.as<uint64_t>(),
                         (int)eimp_W(ctx->i_Mref), ctx->i_sinfo.as<int2>(), ctx->i_phased.as<uint64_t>(), (int)eimp_W(M),
                         ctx->i_gt.as<uint8_t>(), (int)M, (int)nimp, hapmap, (int)mref_begin, (int)nsites,
                         ctx->i_imputeCalls, d_dos, (int)ldd, d_bits, (int)ldb_words, ctx->shape_dos_span,
                         ctx->stream));
    return 0;
}

int eimp_imp_bunch(eimp_ctx *ctx, size_t mref_begin, size_t nsites, uint64_t *bits, float *dos) {
    if (!ctx || !bits || !dos) return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch: NULL argument");
    if (!ctx->i_ntargets) return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch: imputation not prepared");
    if (int r = use_device(ctx)) return r;
    const size_t nh = 2 * ctx->i_ntargets, wb = eimp_W(nsites);
    CK(ctx->i_bits.reserve(nh * wb * 8));
    CK(ctx->i_dos.reserve(nh * nsites * 4));
    CK(cudaMemsetAsync(ctx->i_bits.p, 0, nh * wb * 8, ctx->stream));
    // rows of haploid targets' second haplotype are not imputed: zero
    if (ctx->i_tgthap_n) CK(cudaMemsetAsync(ctx->i_dos.p, 0, nh * nsites * 4, ctx->stream));
    int r = eimp_imp_bunch_dev(ctx, mref_begin, nsites, ctx->i_bits.as<uint64_t>(), wb, ctx->i_dos.as<float>(), nsites);
    if (r) return r;
    CK(cudaMemcpyAsync(bits, ctx->i_bits.p, nh * wb * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(dos, ctx->i_dos.p, nh * nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int eimp_imp_phased_dosages(eimp_ctx *ctx, const float *dos_mat, const float *dos_pat) {
    if (!ctx || !dos_mat || !dos_pat) return fail(ctx, EIMP_E_ARG, "eimp_imp_phased_dosages: NULL argument");
    if (!ctx->i_ntargets) return fail(ctx, EIMP_E_ARG, "eimp_imp_phased_dosages: imputation not prepared");
    if (int r = use_device(ctx)) return r;
    const size_t bytes = ctx->i_ntargets * ctx->i_M * 4;
    CK(ctx->i_pdm.reserve(bytes));
    CK(ctx->i_pdp.reserve(bytes));
    CK(cudaMemcpyAsync(ctx->i_pdm.p, dos_mat, bytes, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->i_pdp.p, dos_pat, bytes, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->i_have_pdos = true;
    return 0;
}

int eimp_imp_site_stats_dev(eimp_ctx *ctx, size_t mref_begin, size_t nsites, const uint64_t *d_bits,
                            size_t ldb_words, const float *d_dos, size_t ldd, const float *d_pdos_mat,
                            const float *d_pdos_pat, size_t ldp, const eimp_site_stats_opts *opts, float *d_ads,
                            size_t lda, uint64_t *d_gtbits, size_t ldg_words, float *d_ds, float *d_gp,
                            float *d_r2, float *d_af, float *d_maf, int32_t *d_ac, int32_t *d_an, uint8_t *d_pass,
                            uint64_t *d_conflicts) {
    if (!ctx || !ctx->i_ntargets) return fail(ctx, EIMP_E_ARG, "eimp_imp_site_stats: imputation not prepared");
    if (!opts || !d_bits || !d_dos || !d_ads || !d_gtbits || !d_r2 || !d_af || !d_maf || !d_ac || !d_an || !d_pass ||
        !d_conflicts)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_site_stats: NULL argument");
    if (mref_begin + nsites > ctx->i_Mref || !nsites) return fail(ctx, EIMP_E_ARG, "eimp_imp_site_stats: window out of range");
    const size_t wb = (nsites + 63) / 64;
    if (ldb_words < wb || ldg_words < wb || ldd < nsites || lda < nsites)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_site_stats: leading dimension too small");
    const float *pm = d_pdos_mat ? d_pdos_mat : (ctx->i_have_pdos ? ctx->i_pdm.as<float>() : nullptr);
    const float *pp = d_pdos_pat ? d_pdos_pat : (ctx->i_have_pdos ? ctx->i_pdp.as<float>() : nullptr);
    if (!d_pdos_mat) ldp = ctx->i_M;
    if (!pm || !pp || ldp < ctx->i_M)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_site_stats: no phased dosages (eimp_imp_phased_dosages)");
    if (int r = use_device(ctx)) return r;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ref_ready, 0));
    SiteStatsArgs a;
    a.ntgt = (int)ctx->i_ntargets; a.mref_begin = (int)mref_begin; a.nsites = (int)nsites;
    a.bits = d_bits; a.ldb = (int)ldb_words; a.dos = d_dos; a.ldd = (int)ldd;
    a.phased = ctx->i_phased.as<uint64_t>(); a.wM = (int)eimp_W(ctx->i_M);
    a.pdos_mat = pm; a.pdos_pat = pp; a.ldp = (int)ldp;
    a.gt = ctx->i_gt.as<uint8_t>(); a.M = (int)ctx->i_M;
    a.segm = ctx->i_segm.as<int32_t>(); a.common = ctx->i_common.as<uint8_t>(); a.af = ctx->i_af.as<float>();
    a.overwriteCalls = opts->overwriteCalls; a.improveCalls = opts->improveCalls;
    a.r2filter = opts->r2filter; a.maffilter = opts->maffilter;
    a.ads = d_ads; a.lda = (int)lda; a.gtbits = d_gtbits; a.ldg = (int)ldg_words; a.ds = d_ds; a.gp = d_gp;
    a.r2 = d_r2; a.af_out = d_af; a.maf = d_maf; a.ac = d_ac; a.an = d_an; a.pass = d_pass;
    a.conflicts = reinterpret_cast<unsigned long long *>(d_conflicts);
    a.haptgt = ctx->i_tgthap_n ? ctx->i_tgtflag.as<uint8_t>() : nullptr;
    a.icnt = opts->improveCalls ? ctx->s_improve.as<unsigned long long>() : nullptr;
    a.itot = opts->improveCalls ? reinterpret_cast<double *>(ctx->s_improve.as<unsigned long long>() + 5) : nullptr;
    LAUNCH(launch_site_stats(a, ctx->stream));
    return 0;
}

int eimp_imp_improve_stats(eimp_ctx *ctx, uint64_t *counts, double *totals, int reset) {
    if (!ctx || !counts || !totals) return fail(ctx, EIMP_E_ARG, "eimp_imp_improve_stats: NULL argument");
    if (int r = use_device(ctx)) return r;
    CK(cudaMemcpyAsync(counts, ctx->s_improve.p, 40, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(totals, ctx->s_improve.as<uint8_t>() + 40, 40, cudaMemcpyDeviceToHost, ctx->stream));
    if (reset) CK(cudaMemsetAsync(ctx->s_improve.p, 0, 80, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int eimp_imp_bunch_stats(eimp_ctx *ctx, size_t mref_begin, size_t nsites, const eimp_site_stats_opts *opts,
                         float *ads, uint64_t *gtbits, float *ds, float *gp, float *r2, float *af, float *maf,
                         int32_t *ac, int32_t *an, uint8_t *pass, uint64_t *conflicts) {
    if (!ctx || !opts || !ads || !gtbits || !r2 || !af || !maf || !ac || !an || !pass || !conflicts)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch_stats: NULL argument");
    if (!ctx->i_ntargets) return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch_stats: imputation not prepared");
    if (!ctx->i_have_pdos) return fail(ctx, EIMP_E_ARG, "eimp_imp_bunch_stats: no phased dosages (eimp_imp_phased_dosages)");
    if (int r = use_device(ctx)) return r;
    const size_t N = ctx->i_ntargets, nh = 2 * N, wb = eimp_W(nsites);
    CK(ctx->i_bits.reserve(nh * wb * 8));
    CK(ctx->i_dos.reserve(nh * nsites * 4));
    CK(ctx->s_ads.reserve(nh * nsites * 4));
    CK(ctx->s_gt.reserve(nh * wb * 8));
    if (ds) CK(ctx->s_ds.reserve(N * nsites * 4));
    if (gp) CK(ctx->s_gp.reserve(3 * N * nsites * 4));
    const size_t site_bytes = nsites * (4 * 3 + 4 * 2 + 1) + 64;
    CK(ctx->s_site.reserve(site_bytes));
    CK(ctx->s_conf.reserve(8));
    CK(cudaMemsetAsync(ctx->i_bits.p, 0, nh * wb * 8, ctx->stream));
    CK(cudaMemsetAsync(ctx->s_gt.p, 0, nh * wb * 8, ctx->stream));
    CK(cudaMemsetAsync(ctx->s_conf.p, 0, 8, ctx->stream));
    int r = eimp_imp_bunch_dev(ctx, mref_begin, nsites, ctx->i_bits.as<uint64_t>(), wb, ctx->i_dos.as<float>(), nsites);
    if (r) return r;
    uint8_t *sb = ctx->s_site.as<uint8_t>();
    float *d_r2 = reinterpret_cast<float *>(sb), *d_af = d_r2 + nsites, *d_maf = d_af + nsites;
    int32_t *d_ac = reinterpret_cast<int32_t *>(d_maf + nsites), *d_an = d_ac + nsites;
    uint8_t *d_pass = reinterpret_cast<uint8_t *>(d_an + nsites);
    r = eimp_imp_site_stats_dev(ctx, mref_begin, nsites, ctx->i_bits.as<uint64_t>(), wb, ctx->i_dos.as<float>(), nsites,
                                nullptr, nullptr, 0, opts, ctx->s_ads.as<float>(), nsites, ctx->s_gt.as<uint64_t>(), wb,
                                ds ? ctx->s_ds.as<float>() : nullptr, gp ? ctx->s_gp.as<float>() : nullptr, d_r2, d_af,
                                d_maf, d_ac, d_an, d_pass, ctx->s_conf.as<uint64_t>());
    if (r) return r;
    CK(cudaMemcpyAsync(ads, ctx->s_ads.p, nh * nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(gtbits, ctx->s_gt.p, nh * wb * 8, cudaMemcpyDeviceToHost, ctx->stream));
    if (ds) CK(cudaMemcpyAsync(ds, ctx->s_ds.p, N * nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (gp) CK(cudaMemcpyAsync(gp, ctx->s_gp.p, 3 * N * nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(r2, d_r2, nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(af, d_af, nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(maf, d_maf, nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(ac, d_ac, nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(an, d_an, nsites * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(pass, d_pass, nsites, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(conflicts, ctx->s_conf.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int eimp_phase_exclude_self(eimp_ctx *ctx, int64_t first_sample) {
    if (!ctx) return EIMP_E_ARG;
    if (first_sample >= 0 && (size_t)first_sample >= ctx->p_nhaps / 2)
        return fail(ctx, EIMP_E_ARG, "eimp_phase_exclude_self: sample outside the phasing reference");
    ctx->self0 = first_sample < 0 ? -1 : first_sample;
    return 0;
}

int eimp_phase_start_phases(eimp_ctx *ctx, size_t ntgt, const uint8_t *phases) {
    if (!ctx || (ntgt && !phases)) return fail(ctx, EIMP_E_ARG, "eimp_phase_start_phases: NULL argument");
    if (int r = use_device(ctx)) return r;
    if (ntgt) {
        CK(ctx->startph.reserve(ntgt));
        CK(cudaMemcpyAsync(ctx->startph.p, phases, ntgt, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    ctx->startph_n = ntgt;
    return 0;
}

int eimp_phase_set_haploid_ref(eimp_ctx *ctx, size_t nsamples, const uint8_t *haploid) {
    if (!ctx) return EIMP_E_ARG;
    if (!ctx->p_M) return fail(ctx, EIMP_E_ARG, "eimp_phase_set_haploid_ref: phasing reference not set");
    if (haploid && 2 * nsamples != ctx->p_nhaps)
        return fail(ctx, EIMP_E_ARG, "eimp_phase_set_haploid_ref: one flag per sample of the phasing reference");
    if (int r = use_device(ctx)) return r;
    size_t n = 0;
    for (size_t i = 0; haploid && i < nsamples; i++) n += haploid[i] != 0;
    if (n) {
        CK(cudaStreamSynchronize(ctx->stream));   // the flags may be in use by queued phasing work
        CK(ctx->p_haploid.reserve(nsamples));
        std::vector<uint8_t> f(haploid, haploid + nsamples);
        for (auto &x : f) x = x != 0;
        CK(cudaMemcpy(ctx->p_haploid.p, f.data(), nsamples, cudaMemcpyHostToDevice));
    }
    ctx->p_nhaploid = n;
    return 0;
}

int eimp_phase_haploid_targets(eimp_ctx *ctx, size_t ntgt, const uint8_t *haploid) {
    if (!ctx || (ntgt && !haploid)) return fail(ctx, EIMP_E_ARG, "eimp_phase_haploid_targets: NULL argument");
    if (int r = use_device(ctx)) return r;
    size_t n = 0;
    for (size_t i = 0; i < ntgt; i++) n += haploid[i] != 0;
    if (n) {
        CK(cudaStreamSynchronize(ctx->stream));
        CK(ctx->tgthap.reserve(ntgt));
        std::vector<uint8_t> f(haploid, haploid + ntgt);
        for (auto &x : f) x = x != 0;
        CK(cudaMemcpy(ctx->tgthap.p, f.data(), ntgt, cudaMemcpyHostToDevice));
    }
    ctx->tgthap_n = n ? ntgt : 0;
    return 0;
}

int eimp_qref_index(const uint8_t *section, size_t nbytes, size_t Mref, size_t Nref, int64_t *offsets) {
    if ((!section && nbytes) || (!offsets && Mref)) return EIMP_E_ARG;
    const size_t raw = eimp_W(2 * Nref) * 8;   // hapcapacity: 2*Nref bits in 512-bit units
    size_t off = 0;
    for (size_t v = 0; v < Mref; v++) {
        if (off + 8 > nbytes) return EIMP_E_ARG;   // "Failed reading haplotypes from reference."
        uint64_t encsize;
        memcpy(&encsize, section + off, 8);
        offsets[v] = (int64_t)off;
        const size_t len = encsize ? encsize : raw;
        if (len > nbytes - off - 8) return EIMP_E_ARG;
        off += 8 + len;
    }
    return 0;
}

int eimp_qref_decode_dev(eimp_ctx *ctx, const uint8_t *d_section, const int64_t *d_offsets, size_t Mref,
                         size_t Nref, uint64_t *d_out, size_t ldw_words) {
    if (!ctx || (Mref && (!d_section || !d_offsets || !d_out))) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode: NULL argument");
    const size_t nw = eimp_W(2 * Nref);
    if (ldw_words < nw) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode: leading dimension too small");
    if (Mref > (size_t)INT32_MAX || nw > (size_t)INT32_MAX) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode: too many variants");
    if (int r = use_device(ctx)) return r;
    LAUNCH(launch_qref_decode(d_section, d_offsets, (int)Mref, (int)nw, d_out, ldw_words, ctx->status.as<uint32_t>(),
                              ctx->stream));
    return 0;
}

int eimp_qref_decode(eimp_ctx *ctx, const uint8_t *section, size_t nbytes, size_t Mref, size_t Nref,
                     uint64_t *d_out, size_t ldw_words, uint64_t *host_out) {
    if (!ctx || (!section && nbytes)) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode: NULL argument");
    const size_t nw = eimp_W(2 * Nref);
    if (!d_out) ldw_words = nw;
    if (ldw_words < nw) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode: leading dimension too small");
    std::vector<int64_t> offs(Mref);
    if (eimp_qref_index(section, nbytes, Mref, Nref, offs.data()))
        return fail(ctx, EIMP_E_ARG, "Failed reading haplotypes from reference.");
    if (int r = use_device(ctx)) return r;
    // the decoder reads whole aligned 32-bit words: 16 bytes of slack past the section
    CK(ctx->q_sec.reserve(nbytes + 16));
    CK(ctx->q_offs.reserve(Mref * 8 + 8));
    CK(cudaMemsetAsync(ctx->q_sec.as<uint8_t>() + nbytes, 0, 16, ctx->stream));
    CK(cudaMemcpyAsync(ctx->q_sec.p, section, nbytes, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->q_offs.p, offs.data(), Mref * 8, cudaMemcpyHostToDevice, ctx->stream));
    uint64_t *dst = d_out;
    if (!dst) {
        CK(ctx->q_out.reserve(Mref * nw * 8 + 8));
        dst = ctx->q_out.as<uint64_t>();
    }
    int r = eimp_qref_decode_dev(ctx, ctx->q_sec.as<uint8_t>(), ctx->q_offs.as<int64_t>(), Mref, Nref, dst, ldw_words);
    if (r) return r;
    if (host_out) {
        if (ldw_words == nw) {
            CK(cudaMemcpyAsync(host_out, dst, Mref * nw * 8, cudaMemcpyDeviceToHost, ctx->stream));
        } else {
            CK(cudaMemcpy2DAsync(host_out, nw * 8, dst, ldw_words * 8, nw * 8, Mref, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

int eimp_qref_decode_masked(eimp_ctx *ctx, const uint8_t *section, size_t nbytes, size_t Mref, size_t Nref,
                            size_t nmasked, const int64_t *masked, const uint8_t *masked_haploid,
                            size_t nhaploid_ref, float *af, uint64_t *d_out, size_t ldw_words, uint64_t *host_out) {
    if (!ctx || (!section && nbytes) || (nmasked && (!masked || !masked_haploid)) || (Mref && !af))
        return fail(ctx, EIMP_E_ARG, "eimp_qref_decode_masked: NULL argument");
    if (nmasked >= Nref) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode_masked: every sample masked");
    size_t mhap = 0;
    for (size_t i = 0; i < nmasked; i++) {
        if (masked[i] < 0 || (size_t)masked[i] >= Nref || (i && masked[i] <= masked[i - 1]))
            return fail(ctx, EIMP_E_ARG, "eimp_qref_decode_masked: masked samples must be ascending sample indices");
        mhap += masked_haploid[i] != 0;
    }
    if (mhap > nhaploid_ref) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode_masked: more haploid samples masked than exist");
    const size_t nw = eimp_W(2 * Nref), nout = Nref - nmasked, nwo = eimp_W(2 * nout);
    if (!d_out) ldw_words = nwo;
    if (ldw_words < nwo) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode_masked: leading dimension too small");
    if (Mref > (size_t)INT32_MAX || nw > (size_t)INT32_MAX) return fail(ctx, EIMP_E_ARG, "eimp_qref_decode_masked: too large");
    std::vector<int64_t> offs(Mref);
    if (eimp_qref_index(section, nbytes, Mref, Nref, offs.data()))
        return fail(ctx, EIMP_E_ARG, "Failed reading haplotypes from reference.");
    std::vector<int32_t> kept;
    kept.reserve(nout);
    for (size_t sIdx = 0, i = 0; sIdx < Nref; sIdx++) {
        if (i < nmasked && (size_t)masked[i] == sIdx) { i++; continue; }
        kept.push_back((int32_t)sIdx);
    }
    if (int r = use_device(ctx)) return r;
    CK(ctx->q_sec.reserve(nbytes + 16));
    CK(ctx->q_offs.reserve(Mref * 8 + 8));
    CK(ctx->q_mask.reserve(nmasked * 8 + 8));
    CK(ctx->q_maskhap.reserve(nmasked + 8));
    CK(ctx->q_kept.reserve(nout * 4 + 8));
    CK(ctx->q_af.reserve(Mref * 4 + 8));
    CK(cudaMemsetAsync(ctx->q_sec.as<uint8_t>() + nbytes, 0, 16, ctx->stream));
    CK(cudaMemcpyAsync(ctx->q_sec.p, section, nbytes, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->q_offs.p, offs.data(), Mref * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (nmasked) {
        CK(cudaMemcpyAsync(ctx->q_mask.p, masked, nmasked * 8, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaMemcpyAsync(ctx->q_maskhap.p, masked_haploid, nmasked, cudaMemcpyHostToDevice, ctx->stream));
    }
    CK(cudaMemcpyAsync(ctx->q_kept.p, kept.data(), nout * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->q_af.p, af, Mref * 4, cudaMemcpyHostToDevice, ctx->stream));
    uint64_t *dst = d_out;
    if (!dst) {
        CK(ctx->q_out.reserve(Mref * nwo * 8 + 8));
        dst = ctx->q_out.as<uint64_t>();
    }
    // the unmasked rows of a chunk of variants, then their masked rows
    const size_t chunk = std::max<size_t>(1, std::min<size_t>(Mref, (size_t(256) << 20) / (nw * 8)));
    CK(ctx->q_rows.reserve(chunk * nw * 8));
    const float an_before = (float)(2 * Nref - nhaploid_ref), an_after = (float)(2 * nout - (nhaploid_ref - mhap));
    for (size_t v0 = 0; v0 < Mref; v0 += chunk) {
        const int n = (int)std::min(chunk, Mref - v0);
        LAUNCH(launch_qref_decode(ctx->q_sec.as<uint8_t>(), ctx->q_offs.as<int64_t>() + v0, n, (int)nw,
                                  ctx->q_rows.as<uint64_t>(), nw, ctx->status.as<uint32_t>(), ctx->stream));
        LAUNCH(launch_qref_mask(ctx->q_sec.as<uint8_t>(), ctx->q_offs.as<int64_t>() + v0, n,
                                ctx->q_rows.as<uint64_t>(), nw, ctx->q_kept.as<int32_t>(), (int)nout, (int)nwo,
                                ctx->q_mask.as<int64_t>(), (int)nmasked, ctx->q_maskhap.as<uint8_t>(), an_before,
                                an_after, ctx->q_af.as<float>() + v0, dst + v0 * ldw_words, ldw_words, ctx->stream));
    }
    CK(cudaMemcpyAsync(af, ctx->q_af.p, Mref * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (host_out) {
        if (ldw_words == nwo) {
            CK(cudaMemcpyAsync(host_out, dst, Mref * nwo * 8, cudaMemcpyDeviceToHost, ctx->stream));
        } else {
            CK(cudaMemcpy2DAsync(host_out, nwo * 8, dst, ldw_words * 8, nwo * 8, Mref, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        }
    }
    CK(cudaStreamSynchronize(ctx->stream));
    return check_status(ctx);
}

int eimp_imp_matches(eimp_ctx *ctx, size_t hap, int32_t *out, size_t cap, size_t *n) {
    if (!ctx || !n || hap >= 2 * ctx->i_ntargets) return fail(ctx, EIMP_E_ARG, "eimp_imp_matches: bad haplotype");
    if (int r = use_device(ctx)) return r;
    int cnt = 0;
    CK(cudaMemcpyAsync(&cnt, ctx->i_nmatch.as<int>() + hap, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (cnt < 0) return fail(ctx, EIMP_E_CAPACITY, "eimp_imp_matches: match search overflowed for this haplotype");
    *n = (size_t)cnt;
    if (out && cnt) {
        size_t k = (size_t)cnt < cap ? (size_t)cnt : cap;
        CK(cudaMemcpyAsync(out, ctx->i_matches.as<int4>() + hap * ctx->i_cap, k * sizeof(int4), cudaMemcpyDeviceToHost,
                           ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    return 0;
}

int eimp_imp_refpbwt(eimp_ctx *ctx, uint32_t *compr, int32_t *absperm) {
    if (!ctx || !ctx->i_Mref) return fail(ctx, EIMP_E_ARG, "eimp_imp_refpbwt: no reference set");
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->i_M, K = ctx->i_K;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ref_ready, 0));
    if (compr) CK(cudaMemcpyAsync(compr, ctx->i_compr.p, M * eimp_kw(K) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (absperm) CK(cudaMemcpyAsync(absperm, ctx->i_absperm.p, (M + 1) * K * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int eimp_imp_prefix_slice(eimp_ctx *ctx, size_t site, size_t lo, size_t hi, int32_t *out) {
    if (!ctx || !ctx->i_Mref) return fail(ctx, EIMP_E_ARG, "eimp_imp_prefix_slice: no reference set");
    if (!out || site > ctx->i_M || lo > hi || hi >= ctx->i_K)
        return fail(ctx, EIMP_E_ARG, "eimp_imp_prefix_slice: slice outside the prefix arrays");
    if (int r = use_device(ctx)) return r;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ref_ready, 0));
    CK(cudaMemcpyAsync(out, ctx->i_absperm.as<int32_t>() + site * ctx->i_K + lo, (hi - lo + 1) * 4,
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int eimp_transpose_bits_dev(eimp_ctx *ctx, const uint64_t *d_src, size_t rows, size_t src_ld, uint64_t *d_dst,
                            size_t cols, size_t dst_ld) {
    if (!ctx || !d_src || !d_dst || src_ld < (cols + 63) / 64 || dst_ld < (rows + 63) / 64 || (cols + 63) / 64 > 65535)
        return fail(ctx, EIMP_E_ARG, "eimp_transpose_bits_dev: bad sizes");
    if (int r = use_device(ctx)) return r;
    LAUNCH(launch_transpose_ld(d_src, rows, src_ld, d_dst, cols, (rows + 63) / 64, dst_ld, ctx->stream));
    return 0;
}

// --------------------------------------------------------------------- phasing

int eimp_phase_set_reference(eimp_ctx *ctx, size_t M, size_t nhaps, const uint64_t *hapmajor,
                             const uint64_t *sitemajor, const float *cM) {
    if (!ctx || !M || !nhaps || !hapmajor || !sitemajor || !cM)
        return fail(ctx, EIMP_E_ARG, "eimp_phase_set_reference: bad argument");
    if (int r = use_device(ctx)) return r;
    const size_t wM = eimp_W(M), wN = eimp_W(nhaps);
    ctx->p_M = M; ctx->p_nhaps = nhaps;
    ctx->p_nhaploid = 0;   // a new panel: all samples diploid until eimp_phase_set_haploid_ref
    CK(ctx->p_hapmajor.reserve(nhaps * wM * 8));
    CK(ctx->p_sitemajor.reserve(M * wN * 8));
    CK(ctx->p_cm.reserve(M * 4));
    CK(cudaMemcpyAsync(ctx->p_hapmajor.p, hapmajor, nhaps * wM * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->p_sitemajor.p, sitemajor, M * wN * 8, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->p_cm.p, cM, M * 4, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

int eimp_phase_set_reference_dev(eimp_ctx *ctx, size_t M, size_t nhaps, const uint64_t *d_sitemajor_full,
                                 size_t ldw_words, const int64_t *d_typed, const float *d_cM) {
    if (!ctx || !M || !nhaps || !d_sitemajor_full || !d_typed || !d_cM)
        return fail(ctx, EIMP_E_ARG, "eimp_phase_set_reference_dev: bad argument");
    const size_t wM = eimp_W(M), wN = eimp_W(nhaps);
    if (ldw_words < wN) return fail(ctx, EIMP_E_ARG, "eimp_phase_set_reference_dev: leading dimension too small");
    if (int r = use_device(ctx)) return r;
    cudaStream_t st = ctx->stream;
    ctx->p_M = M; ctx->p_nhaps = nhaps;
    ctx->p_nhaploid = 0;
    CK(ctx->p_hapmajor.reserve(nhaps * wM * 8));
    CK(ctx->p_sitemajor.reserve(M * wN * 8));
    CK(ctx->p_cm.reserve(M * 4));
    LAUNCH(launch_gather_rows(d_sitemajor_full, ldw_words, d_typed, (int)M, (int)wN, ctx->p_sitemajor.as<uint64_t>(),
                              st));
    CK(cudaMemsetAsync(ctx->p_hapmajor.p, 0, nhaps * wM * 8, st));
    LAUNCH(launch_transpose(ctx->p_sitemajor.as<uint64_t>(), M, wN, ctx->p_hapmajor.as<uint64_t>(), nhaps, wM, st));
    CK(cudaMemcpyAsync(ctx->p_cm.p, d_cM, M * 4, cudaMemcpyDeviceToDevice, st));
    return 0;
}

namespace {

// device-side prepPhase for ntgt targets whose genotypes are at d_gt
int run_prep(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *d_gt) {
    const size_t M = ctx->p_M, nh = ctx->p_nhaps, wM = eimp_W(M), wN = eimp_W(nh);
    const size_t K = phase_K(ctx, p);
    if (ctx->self0 >= 0 && (size_t)ctx->self0 + ntgt > nh / 2)
        return fail(ctx, EIMP_E_ARG, "the batch's own samples lie outside the phasing reference");
    cudaStream_t st = ctx->stream;
    CK(ctx->b_nerr.reserve(ntgt * nh * 4));
    CK(ctx->b_bh.reserve(ntgt * K * 4));
    CK(ctx->b_flags.reserve(ntgt * wN * 8));
    CK(ctx->b_monos.reserve(ntgt * wM * 8));
    CK(ctx->b_splits.reserve(ntgt * M * 4));
    CK(ctx->b_calls.reserve(ntgt * M * 4));
    CK(ctx->b_cmd.reserve(ntgt * (M + 1) * 4));
    CK(ctx->b_nsplits.reserve(ntgt * 4));
    CK(ctx->b_ncalls.reserve(ntgt * 4));
    if (ctx->tgthap_n && ctx->tgthap_n != ntgt)
        return fail(ctx, EIMP_E_ARG, "haploid targets were set for a different number of targets");
    const uint8_t *refhap = ctx->p_nhaploid ? ctx->p_haploid.as<uint8_t>() : nullptr;
    const uint8_t *tgthap = ctx->tgthap_n ? ctx->tgthap.as<uint8_t>() : nullptr;
    LAUNCH(launch_besthaps(d_gt, (int)ntgt, (int)M, ctx->p_hapmajor.as<uint64_t>(), (int)nh, (int)wM, (int)K,
                           ctx->b_nerr.as<uint32_t>(), ctx->b_bh.as<int32_t>(), ctx->b_flags.as<uint64_t>(), (int)wN,
                           (int)ctx->self0, refhap, st));
    LAUNCH(launch_monos_calls(d_gt, (int)ntgt, (int)M, ctx->p_hapmajor.as<uint64_t>(), (int)wM,
                              ctx->b_bh.as<int32_t>(), (int)K, ctx->p_cm.as<float>(), p->cMmaxsplit,
                              ctx->b_monos.as<uint64_t>(), ctx->b_splits.as<int32_t>(), ctx->b_calls.as<int32_t>(),
                              ctx->b_cmd.as<float>(), ctx->b_nsplits.as<int32_t>(), ctx->b_ncalls.as<int32_t>(),
                              tgthap, st));
    return 0;
}

// condensed reference + PBWT for the prepared batch; fills ctx->b_rows and the
// host copy of the row offsets
int run_cref_pbwt(eimp_ctx *ctx, size_t K, size_t ntgt, const uint8_t *d_gt, std::vector<int64_t> &rowoff) {
    const size_t M = ctx->p_M, nh = ctx->p_nhaps, wK = eimp_W(K), kw = eimp_kw(K);
    cudaStream_t st = ctx->stream;
    size_t rows;
    if (ctx->rows_cap > 0) {
        // capacity mode: no host round trip; the offsets are scanned on the
        // device and the kernels skip the batch when it needs more rows
        rows = (size_t)ctx->rows_cap;
        CK(ctx->skipbuf.reserve(sizeof(int)));
        CK(ctx->b_rowoff.reserve((ntgt + 1) * 8));
        LAUNCH(launch_rowoff(ctx->b_nsplits.as<int32_t>(), (int)ntgt, ctx->b_rowoff.as<int64_t>(), ctx->rows_cap,
                             ctx->skipbuf.as<int>(), ctx->status.as<uint32_t>(), st));
        ctx->cur_skip = ctx->skipbuf.as<int>();
        ctx->b_rows = 0;   // not known on the host
        rowoff.clear();
    } else {
        std::vector<int32_t> ns(ntgt);
        CK(cudaMemcpyAsync(ns.data(), ctx->b_nsplits.p, ntgt * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        rowoff.assign(ntgt + 1, 0);
        for (size_t t = 0; t < ntgt; t++) rowoff[t + 1] = rowoff[t] + 2 * (int64_t)ns[t] + 1;
        rows = (size_t)rowoff[ntgt];
        ctx->b_rows = rows;
        ctx->cur_skip = nullptr;
        CK(ctx->b_rowoff.reserve((ntgt + 1) * 8));
        CK(cudaMemcpyAsync(ctx->b_rowoff.p, rowoff.data(), (ntgt + 1) * 8, cudaMemcpyHostToDevice, st));
    }
    CK(ctx->b_cref.reserve(rows * wK * 8));
    CK(ctx->b_count0.reserve(rows * 4));
    CK(ctx->b_pbwt.reserve(2 * rows * kw * 4));
    tmark(ctx, 2);
    LAUNCH(launch_cref(d_gt, (int)ntgt, (int)M, ctx->p_hapmajor.as<uint64_t>(), (int)eimp_W(M), (int)nh,
                       ctx->b_bh.as<int32_t>(), (int)K, ctx->b_splits.as<int32_t>(), ctx->b_nsplits.as<int32_t>(),
                       ctx->b_rowoff.as<int64_t>(), ctx->b_cref.as<uint64_t>(), ctx->cur_skip, st));
    tmark(ctx, 3);
    LAUNCH(launch_pbwt(ctx->b_cref.as<uint64_t>(), ctx->b_count0.as<int32_t>(), ctx->b_rowoff.as<int64_t>(),
                       (int)ntgt, (int)K, ctx->b_pbwt.as<uint32_t>(), kw, 0, ctx->cur_skip, st));
    return 0;
}

int check_phase_args(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt) {
    if (!ctx) return EIMP_E_ARG;
    if (!ctx->p_M) return fail(ctx, EIMP_E_ARG, "phasing reference not set");
    if (!p || p->K <= 0 || !ntgt) return fail(ctx, EIMP_E_ARG, "bad phasing parameters or empty batch");
    if (p->hsize <= 0 || p->hsize > 128 || p->hsize_fast <= 0 || p->hsize_fast > 128)
        return fail(ctx, EIMP_E_ARG, "hsize must be in 1..128 (BooleanHistory holds 128 sites)");
    if (phase_K(ctx, p) > 65536)
        return fail(ctx, EIMP_E_ARG, "K must be at most 65536 (the PBWT kernel keeps 16-bit prefix positions)");
    int optin = 0;
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device) == cudaSuccess &&
        (size_t)16 * eimp_W(ctx->p_M) > (size_t)optin)
        return fail(ctx, EIMP_E_CAPACITY, "too many typed sites: a target's genotype vectors do not fit a CTA's shared memory");
    return 0;
}

}  // namespace

int eimp_phase_prep(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *gt, int32_t *besthaps,
                    uint64_t *flags, uint64_t *monos, int32_t *splits, int32_t *calls, float *cmdiffs,
                    int32_t *nsplits, int32_t *ncalls) {
    if (int r = check_phase_args(ctx, p, ntgt)) return r;
    if (!gt) return fail(ctx, EIMP_E_ARG, "eimp_phase_prep: NULL genotypes");
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->p_M, nh = ctx->p_nhaps, wM = eimp_W(M), wN = eimp_W(nh);
    const size_t K = phase_K(ctx, p);
    cudaStream_t st = ctx->stream;
    CK(ctx->b_gt.reserve(ntgt * M));
    CK(cudaMemcpyAsync(ctx->b_gt.p, gt, ntgt * M, cudaMemcpyHostToDevice, st));
    if (int r = run_prep(ctx, p, ntgt, ctx->b_gt.as<uint8_t>())) return r;
    if (besthaps) CK(cudaMemcpyAsync(besthaps, ctx->b_bh.p, ntgt * K * 4, cudaMemcpyDeviceToHost, st));
    if (flags) CK(cudaMemcpyAsync(flags, ctx->b_flags.p, ntgt * wN * 8, cudaMemcpyDeviceToHost, st));
    if (monos) CK(cudaMemcpyAsync(monos, ctx->b_monos.p, ntgt * wM * 8, cudaMemcpyDeviceToHost, st));
    if (splits) CK(cudaMemcpyAsync(splits, ctx->b_splits.p, ntgt * M * 4, cudaMemcpyDeviceToHost, st));
    if (calls) CK(cudaMemcpyAsync(calls, ctx->b_calls.p, ntgt * M * 4, cudaMemcpyDeviceToHost, st));
    if (cmdiffs) CK(cudaMemcpyAsync(cmdiffs, ctx->b_cmd.p, ntgt * (M + 1) * 4, cudaMemcpyDeviceToHost, st));
    if (nsplits) CK(cudaMemcpyAsync(nsplits, ctx->b_nsplits.p, ntgt * 4, cudaMemcpyDeviceToHost, st));
    if (ncalls) CK(cudaMemcpyAsync(ncalls, ctx->b_ncalls.p, ntgt * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

int eimp_phase_cref_pbwt(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *gt,
                         size_t *rows_out, int64_t *rowoff, uint64_t *cref, int32_t *count0, uint32_t *pbwt) {
    if (int r = check_phase_args(ctx, p, ntgt)) return r;
    if (!gt || !rows_out) return fail(ctx, EIMP_E_ARG, "eimp_phase_cref_pbwt: NULL argument");
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->p_M, nh = ctx->p_nhaps;
    const size_t K = phase_K(ctx, p);
    cudaStream_t st = ctx->stream;
    CK(ctx->b_gt.reserve(ntgt * M));
    CK(cudaMemcpyAsync(ctx->b_gt.p, gt, ntgt * M, cudaMemcpyHostToDevice, st));
    if (int r = run_prep(ctx, p, ntgt, ctx->b_gt.as<uint8_t>())) return r;
    std::vector<int64_t> ro;
    if (int r = run_cref_pbwt(ctx, K, ntgt, ctx->b_gt.as<uint8_t>(), ro)) return r;
    if (ctx->rows_cap > 0) {   // offsets were computed on the device
        ro.assign(ntgt + 1, 0);
        CK(cudaMemcpyAsync(ro.data(), ctx->b_rowoff.p, (ntgt + 1) * 8, cudaMemcpyDeviceToHost, st));
        if (int r = check_status(ctx)) return r;
        ctx->b_rows = (size_t)ro[ntgt];
    }
    *rows_out = ctx->b_rows;
    if (rowoff) memcpy(rowoff, ro.data(), (ntgt + 1) * 8);
    if (cref) CK(cudaMemcpyAsync(cref, ctx->b_cref.p, ctx->b_rows * eimp_W(K) * 8, cudaMemcpyDeviceToHost, st));
    if (count0) CK(cudaMemcpyAsync(count0, ctx->b_count0.p, ctx->b_rows * 4, cudaMemcpyDeviceToHost, st));
    if (pbwt) CK(cudaMemcpyAsync(pbwt, ctx->b_pbwt.p, 2 * ctx->b_rows * eimp_kw(K) * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

namespace {

size_t hist_len(int hsize, float hist) {
    // Target.cpp:326,466: static_cast<size_t>((HistorySize * hist) + 0.5)
    return (size_t)((double)((float)hsize * hist) + 0.5);
}

int make_beam_params(eimp_ctx *ctx, const eimp_phase_params *p, size_t K, BeamParams &bp) {
    bp.K = (int)K;
    bp.H = (int)hist_len(p->hsize, p->hist);
    bp.Hf = (int)hist_len(p->hsize_fast, p->hist);
    if (bp.H < 1 || bp.H > 128 || bp.Hf < 1 || bp.Hf > 128)
        return fail(ctx, EIMP_E_ARG, "history length hsize*hist must be in 1..128 (BooleanHistory.cpp:31-37)");
    if (p->beamwidth < 1 || p->beamwidth > 128 || p->beamwidth_fast < 1 || p->beamwidth_fast > 128)
        return fail(ctx, EIMP_E_ARG, "beam width must be in 1..128");
    bp.P = p->beamwidth; bp.Pf = p->beamwidth_fast;
    bp.Delta = p->delta; bp.Deltaf = p->delta_fast;
    bp.expectIBDcM = p->expectIBDcM; bp.pErr = p->pErr; bp.pLimit = p->pLimit;
    bp.minfixsize = p->minfixsize; bp.maxfixsize = p->maxfixsize;
    bp.minfixthr = p->minfixthr; bp.maxfixthr = p->maxfixthr;
    bp.doPrePhasing = p->doPrePhasing; bp.doRevPhasing = p->doRevPhasing;
    return 0;
}

int run_phase(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *d_gt, uint64_t *d_mats,
              uint64_t *d_pats, float *d_dm, float *d_dp, float *d_tc, int32_t *d_nc) {
    const size_t M = ctx->p_M, nh = ctx->p_nhaps;
    const size_t K = phase_K(ctx, p);
    BeamParams bp;
    if (int r = make_beam_params(ctx, p, K, bp)) return r;
    if (ctx->startph_n) {
        if (ctx->startph_n != ntgt)
            return fail(ctx, EIMP_E_ARG, "start phases were set for a different number of targets");
        bp.startph = ctx->startph.as<uint8_t>();
    }
    ctx->tvalid = false;
    tmark(ctx, 0);
    if (int r = run_prep(ctx, p, ntgt, d_gt)) return r;
    tmark(ctx, 1);
    std::vector<int64_t> ro;
    if (int r = run_cref_pbwt(ctx, K, ntgt, d_gt, ro)) return r;
    const size_t ab = beam_arena_bytes(bp, (int)M);
    const int slots = beam_slots(bp, (int)M, (int)ntgt, ctx->shape_beam_pct);
    if (slots < 1) return fail(ctx, EIMP_E_CUDA, "beam launch shape: occupancy query failed");
    CK(ctx->b_arena.reserve((size_t)slots * ab));
    CK(ctx->b_order.reserve(ntgt * sizeof(int32_t)));
    CK(ctx->b_workq.reserve(sizeof(int)));
    tmark(ctx, 4);
    LAUNCH(launch_beam(bp, (int)ntgt, (int)M, d_gt, ctx->b_monos.as<uint64_t>(), ctx->b_splits.as<int32_t>(),
                       ctx->b_nsplits.as<int32_t>(), ctx->b_calls.as<int32_t>(), ctx->b_ncalls.as<int32_t>(),
                       ctx->b_cmd.as<float>(), ctx->b_pbwt.as<uint32_t>(), ctx->b_count0.as<int32_t>(),
                       ctx->b_rowoff.as<int64_t>(), ctx->b_arena.p, ab, slots, ctx->b_order.as<int32_t>(),
                       ctx->b_workq.as<int>(), d_mats, d_pats, d_dm, d_dp, d_tc, d_nc, ctx->status.as<uint32_t>(),
                       ctx->cur_skip, ctx->stream));
    if (ctx->tgthap_n)   // haploid targets are not phased (Target.cpp:166-203)
        LAUNCH(launch_haploid_phase(d_gt, (int)ntgt, (int)M, (int)eimp_W(M), ctx->tgthap.as<uint8_t>(), d_mats,
                                    d_pats, d_dm, d_dp, d_tc, d_nc, ctx->status.as<uint32_t>(), ctx->stream));
    tmark(ctx, 5);
    ctx->tvalid = ctx->timing;
    return 0;
}

}  // namespace

extern "C" {

int eimp_phase_reserve(eimp_ctx *ctx, const eimp_phase_params *p, size_t max_targets, size_t max_rows) {
    if (!max_rows) {   // back to host-sized offsets
        if (!ctx) return EIMP_E_ARG;
        ctx->rows_cap = 0;
        return 0;
    }
    if (int r = check_phase_args(ctx, p, max_targets)) return r;
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->p_M, nh = ctx->p_nhaps, wM = eimp_W(M), wN = eimp_W(nh);
    const size_t K = phase_K(ctx, p);
    BeamParams bp;
    bp.K = (int)K;
    if (int r = make_beam_params(ctx, p, K, bp)) return r;
    const size_t n = max_targets;
    CK(ctx->b_gt.reserve(n * M));
    CK(ctx->b_nerr.reserve(n * nh * 4));
    CK(ctx->b_bh.reserve(n * K * 4));
    CK(ctx->b_flags.reserve(n * wN * 8));
    CK(ctx->b_monos.reserve(n * wM * 8));
    CK(ctx->b_splits.reserve(n * M * 4));
    CK(ctx->b_calls.reserve(n * M * 4));
    CK(ctx->b_cmd.reserve(n * (M + 1) * 4));
    CK(ctx->b_nsplits.reserve(n * 4));
    CK(ctx->b_ncalls.reserve(n * 4));
    CK(ctx->b_rowoff.reserve((n + 1) * 8));
    CK(ctx->b_cref.reserve(max_rows * eimp_W(K) * 8));
    CK(ctx->b_count0.reserve(max_rows * 4));
    CK(ctx->b_pbwt.reserve(2 * max_rows * eimp_kw(K) * 4));
    const int slots = beam_slots(bp, (int)M, (int)n);   // the most any launch shape takes
    if (slots < 1) return fail(ctx, EIMP_E_CUDA, "beam launch shape: occupancy query failed");
    CK(ctx->b_arena.reserve((size_t)slots * beam_arena_bytes(bp, (int)M)));
    CK(ctx->b_order.reserve(n * sizeof(int32_t)));
    CK(ctx->b_workq.reserve(sizeof(int)));
    CK(ctx->skipbuf.reserve(sizeof(int)));
    ctx->rows_cap = (int64_t)max_rows;
    return 0;
}

int eimp_phase_targets_dev(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *d_gt,
                           uint64_t *d_mats, uint64_t *d_pats, float *d_dos_mats, float *d_dos_pats,
                           float *d_totalconf, int32_t *d_ncallsites) {
    if (int r = check_phase_args(ctx, p, ntgt)) return r;
    if (!d_gt || !d_mats || !d_pats || !d_dos_mats || !d_dos_pats || !d_totalconf || !d_ncallsites)
        return fail(ctx, EIMP_E_ARG, "eimp_phase_targets: NULL argument");
    if (int r = use_device(ctx)) return r;
    return run_phase(ctx, p, ntgt, d_gt, d_mats, d_pats, d_dos_mats, d_dos_pats, d_totalconf, d_ncallsites);
}

int eimp_phase_targets(eimp_ctx *ctx, const eimp_phase_params *p, size_t ntgt, const uint8_t *gt, uint64_t *mats,
                       uint64_t *pats, float *dos_mats, float *dos_pats, float *totalconf, int32_t *ncallsites) {
    if (int r = check_phase_args(ctx, p, ntgt)) return r;
    if (!gt || !mats || !pats || !dos_mats || !dos_pats || !totalconf || !ncallsites)
        return fail(ctx, EIMP_E_ARG, "eimp_phase_targets: NULL argument");
    if (int r = use_device(ctx)) return r;
    const size_t M = ctx->p_M, wM = eimp_W(M);
    cudaStream_t st = ctx->stream;
    CK(ctx->b_gt.reserve(ntgt * M));
    CK(ctx->b_out_mat.reserve(ntgt * wM * 8));
    CK(ctx->b_out_pat.reserve(ntgt * wM * 8));
    CK(ctx->b_out_dm.reserve(ntgt * M * 4));
    CK(ctx->b_out_dp.reserve(ntgt * M * 4));
    CK(ctx->b_out_tc.reserve(ntgt * 4));
    CK(ctx->b_out_nc.reserve(ntgt * 4));
    CK(cudaMemcpyAsync(ctx->b_gt.p, gt, ntgt * M, cudaMemcpyHostToDevice, st));
    int r = run_phase(ctx, p, ntgt, ctx->b_gt.as<uint8_t>(), ctx->b_out_mat.as<uint64_t>(),
                      ctx->b_out_pat.as<uint64_t>(), ctx->b_out_dm.as<float>(), ctx->b_out_dp.as<float>(),
                      ctx->b_out_tc.as<float>(), ctx->b_out_nc.as<int32_t>());
    if (r) return r;
    CK(cudaMemcpyAsync(mats, ctx->b_out_mat.p, ntgt * wM * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(pats, ctx->b_out_pat.p, ntgt * wM * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(dos_mats, ctx->b_out_dm.p, ntgt * M * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(dos_pats, ctx->b_out_dp.p, ntgt * M * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(totalconf, ctx->b_out_tc.p, ntgt * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(ncallsites, ctx->b_out_nc.p, ntgt * 4, cudaMemcpyDeviceToHost, st));
    return check_status(ctx);
}

}  // extern "C"

// ------------------------------------------------------------ GPUEngine drop-in

int eimp_gpu_initialize(eimp_ctx *ctx, size_t K, size_t Kwords, size_t M, size_t Nrefhapscorr, size_t NrefhapsAD,
                        size_t refTCapacity, const uint64_t *refTData) {
    if (!ctx || !refTData || !K || !M || !NrefhapsAD || K > NrefhapsAD || Kwords != eimp_W(K) ||
        refTCapacity < eimp_W(NrefhapsAD) * 8 || refTCapacity % 64)
        return fail(ctx, EIMP_E_ARG, "eimp_gpu_initialize: inconsistent sizes");
    if (int r = use_device(ctx)) return r;
    ctx->g_K = K; ctx->g_Kwords = Kwords; ctx->g_M = M; ctx->g_Ncorr = Nrefhapscorr; ctx->g_NAD = NrefhapsAD;
    ctx->g_refTcap = refTCapacity;
    CK(ctx->g_refT.reserve(M * refTCapacity));
    CK(cudaMemcpyAsync(ctx->g_refT.p, refTData, M * refTCapacity, cudaMemcpyHostToDevice, ctx->stream));
    // haplotype-major copy for the condensed-reference kernel
    const size_t wM = eimp_W(M);
    CK(ctx->g_hapT.reserve(NrefhapsAD * wM * 8));
    CK(cudaMemsetAsync(ctx->g_hapT.p, 0, NrefhapsAD * wM * 8, ctx->stream));
    LAUNCH(launch_transpose(ctx->g_refT.as<uint64_t>(), M, refTCapacity / 8, ctx->g_hapT.as<uint64_t>(), NrefhapsAD,
                            wM, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return 0;
}

size_t eimp_gpu_block_size(const eimp_ctx *ctx) { (void)ctx; return 1024; }

}  // extern "C"

namespace eimp {
cudaError_t ensure_dynamic_smem(const void *kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> limit;   // per device and kernel
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t &cur = limit[{dev, kernel}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// unpack the reference GPU path's per-target inputs into genotype bytes,
// split lists and best-haplotype lists (one CTA per target)
__global__ void unpack_gpu_inputs(const uint64_t *__restrict__ gtw, const uint64_t *__restrict__ splitw,
                                  const uint64_t *__restrict__ flagw, int M, int wM, int nhaps, int wN, int K,
                                  uint8_t *__restrict__ gt, int32_t *__restrict__ splits, int32_t *__restrict__ nsplits,
                                  int32_t *__restrict__ bh) {
    const int t = blockIdx.x;
    const uint64_t *g = gtw + (size_t)t * 2 * wM;
    const uint64_t *s = splitw + (size_t)t * wM;
    const uint64_t *f = flagw + (size_t)t * wN;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        int a = (g[2 * (m >> 6)] >> (m & 63)) & 1, b = (g[2 * (m >> 6) + 1] >> (m & 63)) & 1;
        gt[(size_t)t * M + m] = (uint8_t)(a && b ? 3 : (a ? 0 : (b ? 2 : 1)));
    }
    if (threadIdx.x == 0) {
        int n = 0;
        for (int m = 0; m < M; m++) if ((s[m >> 6] >> (m & 63)) & 1) splits[(size_t)t * M + n++] = m;
        nsplits[t] = n;
        int k = 0;
        if (K == nhaps) for (int h = 0; h < nhaps; h++) bh[(size_t)t * K + h] = h;
        else for (int h = 0; h < nhaps && k < K; h++) if ((f[h >> 6] >> (h & 63)) & 1) bh[(size_t)t * K + k++] = h;
    }
}
}  // namespace eimp

extern "C" int eimp_gpu_run_cref_pbwt(eimp_ctx *ctx, size_t ntgt, const uint64_t *const *tgtData,
                                      const uint64_t *const *splitData, const uint64_t *const *besthapData,
                                      const uint32_t *crefTOffsets, uint32_t *const *cPBWT, int *const *count0s) {
    if (!ctx || !ctx->g_M) return fail(ctx, EIMP_E_ARG, "eimp_gpu_run_cref_pbwt: engine not initialized");
    if (!ntgt || ntgt > eimp_gpu_block_size(ctx) || !tgtData || !splitData || !besthapData || !crefTOffsets || !cPBWT ||
        !count0s)
        return fail(ctx, EIMP_E_ARG, "eimp_gpu_run_cref_pbwt: bad arguments");
    if (int r = use_device(ctx)) return r;
    // rows of the uploaded reference and the best-haplotype flags are
    // refTCapacity bytes long (GPUEngine.cu:78)
    const size_t M = ctx->g_M, K = ctx->g_K, nh = ctx->g_NAD, wM = eimp_W(M), wN = ctx->g_refTcap / 8;
    const size_t wK = ctx->g_Kwords, stride = 4 * ctx->g_Kwords;
    const size_t gtbytes = eimp_W(2 * M) * 8;   // tgtGTSize (GPUEngine.cu:76)
    cudaStream_t st = ctx->stream;
    DBuf hgt, hsp, hfl;
    CK(hgt.reserve(ntgt * 2 * wM * 8));
    CK(hsp.reserve(ntgt * wM * 8));
    CK(hfl.reserve(ntgt * wN * 8));
    CK(cudaMemsetAsync(hgt.p, 0, ntgt * 2 * wM * 8, st));
    for (size_t t = 0; t < ntgt; t++) {
        CK(cudaMemcpyAsync(hgt.as<uint64_t>() + t * 2 * wM, tgtData[t], gtbytes, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(hsp.as<uint64_t>() + t * wM, splitData[t], wM * 8, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(hfl.as<uint64_t>() + t * wN, besthapData[t], wN * 8, cudaMemcpyHostToDevice, st));
    }
    CK(ctx->g_gt.reserve(ntgt * M));
    CK(ctx->g_splits.reserve(ntgt * M * 4));
    CK(ctx->g_nsplits.reserve(ntgt * 4));
    CK(ctx->g_bh.reserve(ntgt * K * 4));
    eimp::unpack_gpu_inputs<<<(unsigned)ntgt, 256, 0, st>>>(hgt.as<uint64_t>(), hsp.as<uint64_t>(), hfl.as<uint64_t>(),
                                                             (int)M, (int)wM, (int)nh, (int)wN, (int)K,
                                                             ctx->g_gt.as<uint8_t>(), ctx->g_splits.as<int32_t>(),
                                                             ctx->g_nsplits.as<int32_t>(), ctx->g_bh.as<int32_t>());
    ctx->launches++;
    CK(cudaGetLastError());
    std::vector<int64_t> ro(ntgt + 1);
    for (size_t t = 0; t <= ntgt; t++) ro[t] = crefTOffsets[t];
    const size_t rows = (size_t)ro[ntgt];
    CK(ctx->g_rowoff.reserve((ntgt + 1) * 8));
    CK(ctx->g_cref.reserve(rows * wK * 8));
    CK(ctx->g_count0.reserve(rows * 4));
    CK(ctx->g_pbwt.reserve(2 * rows * stride * 4));
    CK(cudaMemcpyAsync(ctx->g_rowoff.p, ro.data(), (ntgt + 1) * 8, cudaMemcpyHostToDevice, st));
    LAUNCH(launch_cref(ctx->g_gt.as<uint8_t>(), (int)ntgt, (int)M, ctx->g_hapT.as<uint64_t>(), (int)wM, (int)nh,
                       ctx->g_bh.as<int32_t>(), (int)K, ctx->g_splits.as<int32_t>(), ctx->g_nsplits.as<int32_t>(),
                       ctx->g_rowoff.as<int64_t>(), ctx->g_cref.as<uint64_t>(), nullptr, st));
    LAUNCH(launch_pbwt(ctx->g_cref.as<uint64_t>(), ctx->g_count0.as<int32_t>(), ctx->g_rowoff.as<int64_t>(), (int)ntgt,
                       (int)K, ctx->g_pbwt.as<uint32_t>(), stride, 1, nullptr, st));
    for (size_t t = 0; t < ntgt; t++) {
        size_t nr = (size_t)(ro[t + 1] - ro[t]);
        CK(cudaMemcpyAsync(cPBWT[t], ctx->g_pbwt.as<uint32_t>() + 2 * (size_t)ro[t] * stride, 2 * nr * stride * 4,
                           cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(count0s[t], ctx->g_count0.as<int32_t>() + ro[t], nr * 4, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return 0;
}
