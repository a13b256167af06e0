/*
 * Test-oracle driver: a C ABI over the reference's OWN hot-path classes
 * (Target, PBWT, Beam, TargetImp, PBWTImputer), compiled from the read-only
 * reference sources by oracle/Makefile into oracle/_ref/libeimp_refcore.so.
 *
 * This file is test infrastructure written for this project.  It is used by
 * tests/ (to pin the oracle restatement and to make golden fixtures) and by
 * bench.py's CPU-baseline leg; the product never links it.
 *
 * The reference keeps intermediate results in private members; the driver
 * reads them by compiling the reference headers with private/protected
 * mapped to public (only inside this translation unit).
 */
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <cmath>
#include <cassert>
#include <string>
#include <vector>
#include <list>
#include <map>
#include <unordered_map>
#include <array>
#include <utility>
#include <memory>
#include <atomic>
#include <mutex>
#include <functional>
#include <algorithm>
#include <stdexcept>
#include <iostream>
#include <iomanip>
#include <sstream>
#include <fstream>
#include <omp.h>
#include <sys/resource.h>
#include <sys/time.h>

#define private public
#define protected public
#include "VCFData.h"
#include "Target.h"
#include "PBWT.h"
#include "PBWTImputer.h"
#include "TargetImp.h"
#undef private
#undef protected

#include "StatusFile.h"
#include "MyMalloc.h"
#include "utils.h"

StatusFile StatusFile::instance;
MyMalloc MyMalloc::mm;

namespace {

size_t capBytes(size_t nbits) { return roundToMultiple(nbits, UNITWORDS * sizeof(uint64_t) * 8) / 8; }

struct Handle {
    VCFData vd;
    bool lastIter = true;
    // NrefhapsCorrected of PBWTPhaser (PBWTPhaser.cpp:408-476, 630, 681): all
    // haplotypes less one per haploid sample of the panel, and less the
    // target's own two in iterations after the first
    size_t ncorr() const {
        size_t n = vd.Nrefhaps - vd.nHaploidsRef;
        if (vd.NrefhapsOrig) n -= vd.nHaploidsTgt + 2;
        return n;
    }
    std::vector<uint64_t*> bufs;
    ~Handle() { for (auto p : bufs) free(p); }
    uint64_t *alloc(size_t bytes) {
        void *p = aligned_alloc(64, bytes ? bytes : 64);
        memset(p, 0, bytes);
        bufs.push_back((uint64_t*)p);
        return (uint64_t*)p;
    }
};

struct ImpHandle {
    Handle *h;
    std::string statfile;
    PBWTImputer *imp = nullptr;
    std::vector<BooleanVector> phased;
    uint64_t *pdata = nullptr;
    ~ImpHandle() { delete imp; free(pdata); }
};

void setParams(int hsize, int beamwidth, int delta, float cMmaxsplit,
               int hsize_fast, int beamwidth_fast, int delta_fast) {
    Target::cMmaxSplit = cMmaxsplit;
    Target::HistorySize = hsize;
    Target::BeamWidth = beamwidth;
    Target::Delta = delta;
    Target::HistorySizeFast = hsize_fast;
    Target::BeamWidthFast = beamwidth_fast;
    Target::DeltaFast = delta_fast;
    Target::minFixSize = 0.5;
    Target::maxFixSize = 0.9;
    Target::minFixThresh = 0.99;
    Target::maxFixThresh = 1.0;
}

} // namespace

extern "C" {

/* Panel + targets.  Bit matrices are given in the reference's layouts with
 * 512-bit padded rows: hapmajor_typed (nhaps x W(M)), sitemajor_typed
 * (M x W(nhaps)), sitemajor_full (Mref x W(nhaps)); gt is ntarget x M with
 * 0/1/2 and 3 = missing. */
void *refo_create(size_t nhaps, size_t M, size_t Mref,
                  const uint64_t *hapmajor_typed, const uint64_t *sitemajor_typed,
                  const uint64_t *sitemajor_full, const int64_t *typed_idx,
                  const float *cm_typed, const float *af_full, const float *af_common,
                  size_t ntarget, const uint8_t *gt) {
    Handle *h = new Handle();
    VCFData &v = h->vd;
    v.Nrefhaps = nhaps; v.M = M; v.Mref = Mref; v.Ntarget = ntarget;
    size_t capM = capBytes(M), capN = capBytes(nhaps);
    v.reference.resize(nhaps);
    uint64_t *rd = h->alloc(nhaps * capM);
    memcpy(rd, hapmajor_typed, nhaps * capM);
    for (size_t i = 0; i < nhaps; i++) v.reference[i].setData(rd + i * capM / 8, capM, M);
    v.referenceT.reset(M, M);
    uint64_t *rt = h->alloc(M * capN);
    memcpy(rt, sitemajor_typed, M * capN);
    for (size_t m = 0; m < M; m++) v.referenceT[m].setData(rt + m * capN / 8, capN, nhaps);
    v.referenceFullT.resize(Mref);
    uint64_t *rf = h->alloc(Mref * capN);
    memcpy(rf, sitemajor_full, Mref * capN);
    for (size_t m = 0; m < Mref; m++) v.referenceFullT[m].setData(rf + m * capN / 8, capN, nhaps);
    v.cMs.reset(M, M);
    for (size_t m = 0; m < M; m++) v.cMs[m] = cm_typed[m];
    v.indexToRefFull.assign(typed_idx, typed_idx + M);
    v.alleleFreqsFullRefRegion.assign(af_full, af_full + Mref);
    v.alleleFreqsCommon.assign(af_common, af_common + M);
    v.haploidsRef.assign(nhaps / 2, false);
    v.haploidsTgt.assign(ntarget, false);
    v.haploidsRefMap.resize(nhaps);
    for (size_t i = 0; i < nhaps; i++) v.haploidsRefMap[i] = i;
    v.haploidsTgtMap.resize(2 * ntarget);
    for (size_t i = 0; i < 2 * ntarget; i++) v.haploidsTgtMap[i] = i;
    v.chunkStartPhase.assign(ntarget, false);
    v.targets.resize(ntarget);
    v.tgtmiss.resize(ntarget);
    v.tgtinphase.resize(ntarget);
    for (size_t t = 0; t < ntarget; t++) {
        v.targets[t].reserve(M);
        v.tgtmiss[t].reset(16, 0);
        v.targetIDs.push_back("t" + std::to_string(t));
        for (size_t m = 0; m < M; m++) {
            uint8_t g = gt[t * M + m];
            v.targets[t].push_back((Genotype)g);
            if (g == 3) v.tgtmiss[t].push_back(m);
        }
    }
    return h;
}

void refo_destroy(void *hp) { delete (Handle*)hp; }

/* Ploidy of the panel's samples (nhaps/2 bytes) and of the targets (ntarget
 * bytes), 1 = haploid; NULL = all diploid.  Sets what VCFData holds after
 * reading a Qref and the targets (VCFData.cpp:1900-1935, 2157-2209, 1340-1348):
 * haploidsRef/haploidsTgt, their counts, and the index maps of the haplotypes
 * that exist (2i, and 2i+1 for a diploid sample).  In phasing iterations
 * after the first the panel's trailing samples are the targets: their flags
 * come in ref (as the reference sets haploidsRef[Nref+i]) and count as target
 * haploids, not reference ones. */
void refo_set_haploids(void *hp, const uint8_t *ref, const uint8_t *tgt) {
    Handle *h = (Handle*)hp;
    VCFData &v = h->vd;
    const size_t ns = v.Nrefhaps / 2, nref = (v.NrefhapsOrig ? v.NrefhapsOrig : v.Nrefhaps) / 2;
    v.haploidsRef.assign(ns, false);
    v.haploidsRefMap.clear();
    v.nHaploidsRef = 0;
    for (size_t i = 0; i < ns; i++) {
        const bool hap = ref && ref[i];
        v.haploidsRef[i] = hap;
        if (hap && i < nref) v.nHaploidsRef++;
        v.haploidsRefMap.push_back(2 * i);
        if (!hap) v.haploidsRefMap.push_back(2 * i + 1);
    }
    v.haploidsTgt.assign(v.Ntarget, false);
    v.haploidsTgtMap.clear();
    v.nHaploidsTgt = 0;
    for (size_t i = 0; i < v.Ntarget; i++) {
        const bool hap = tgt && tgt[i];
        v.haploidsTgt[i] = hap;
        if (hap) v.nHaploidsTgt++;
        v.haploidsTgtMap.push_back(2 * i);
        if (!hap) v.haploidsTgtMap.push_back(2 * i + 1);
    }
}

/* Start phases of the targets (VCFData::chunkStartPhase, carried over from
 * the previous chunk, VCFData.cpp:2802-2816): ntarget bytes, 0 = Ref. */
void refo_set_start_phases(void *hp, const uint8_t *ph) {
    Handle *h = (Handle*)hp;
    for (size_t t = 0; t < h->vd.chunkStartPhase.size(); t++) h->vd.chunkStartPhase[t] = ph[t] != 0;
}

/* Phasing iteration after the first (PBWTPhaser.cpp:406-476): the handle's
 * panel is the reference (nhaps_orig haplotypes) followed by the phased
 * targets; last_iter as Target's lastIter (reverse phasing and call
 * confidences only in the last iteration). */
void refo_set_iteration(void *hp, size_t nhaps_orig, int last_iter) {
    Handle *h = (Handle*)hp;
    h->vd.NrefhapsOrig = nhaps_orig;
    h->lastIter = last_iter != 0;
}

void refo_set_params(int hsize, int beamwidth, int delta, float cMmaxsplit,
                     int hsize_fast, int beamwidth_fast, int delta_fast) {
    setParams(hsize, beamwidth, delta, cMmaxsplit, hsize_fast, beamwidth_fast, delta_fast);
}

/* Target::prepPhase (Target.cpp:95-163): best haps, monos, split/call sites.
 * Buffers: besthaps K; monos W(M) words; splits/calls/cmdiffs capacity M+1.
 * Returns the number of split sites S (ncalls via *ncalls). */
long refo_prep(void *hp, size_t t, size_t K,
               int64_t *besthaps, uint64_t *monos, int64_t *splitsites,
               int64_t *calllocs, size_t *ncalls, float *cmsplitdiffs) {
    Handle *h = (Handle*)hp;
    VCFData &v = h->vd;
    BooleanVector pm, pp; std::vector<float> dm, dp;
    Target tg(pm, pp, dm, dp, t, v.targetIDs[t], v, v.Nrefhaps, h->ncorr(), K,
              2.0f, 1.0f, 0.003f, 0.003f, false, true, true, false, false, false);
    tg.prepPhase();
    for (size_t k = 0; k < K; k++) besthaps[k] = tg.bestHaps[k];
    memcpy(monos, tg.monos.getData(), capBytes(v.M));
    size_t S = tg.splitsites.size();
    for (size_t s = 0; s < S; s++) splitsites[s] = tg.splitsites[s];
    for (size_t c = 0; c < tg.callLocs.size(); c++) calllocs[c] = tg.callLocs[c];
    *ncalls = tg.callLocs.size();
    for (size_t i = 0; i < tg.cMsplitDiffs.size(); i++) cmsplitdiffs[i] = tg.cMsplitDiffs[i];
    return (long)S;
}

/* Condensed reference + compressed PBWT of one target, CPU path
 * (Target.cpp:248-282, PBWT.cpp:33-70,207-285).
 * cref: (2S+1) x W(K) words; count0: 2S+1; pbwt: 2*(2S+1) rows x 2*ceil(K/32) u32. */
long refo_cref_pbwt(void *hp, size_t t, size_t K, uint64_t *cref, int *count0, uint32_t *pbwt) {
    Handle *h = (Handle*)hp;
    VCFData &v = h->vd;
    BooleanVector pm, pp; std::vector<float> dm, dp;
    Target tg(pm, pp, dm, dp, t, v.targetIDs[t], v, v.Nrefhaps, h->ncorr(), K,
              2.0f, 1.0f, 0.003f, 0.003f, false, true, true, false, false, false);
    tg.prepPhase();
    size_t Mp = 2 * tg.splitsites.size() + 1;
    size_t capacity = capBytes(K);
    uint64_t *refincdata = (uint64_t*)MyMalloc::calloc(Mp * capacity, 1, "refo_refinc");
    RingBuffer<BooleanVector> refincT(Mp, Mp);
    uint64_t *cur = refincdata;
    for (auto &r : refincT) { r.setData(cur, capacity, K); cur += capacity / 8; }
    std::vector<int> *c0 = new std::vector<int>(Mp);
    tg.condensedReferenceT(refincT, c0);
    if (cref) memcpy(cref, refincdata, Mp * capacity);
    if (count0) for (size_t i = 0; i < Mp; i++) count0[i] = (*c0)[i];
    {
        PBWT pb(&refincT, c0, t);   // takes ownership of c0
        if (pbwt) memcpy(pbwt, pb.comprPBWT, 2 * Mp * pb.Kwords * sizeof(uint32_t));
    }
    MyMalloc::free(refincdata);
    return (long)Mp;
}

/* Full phasing of one target: Target::phase() (Target.cpp:166-289).
 * mat/pat: W(M) words each; dos_mat/dos_pat: M floats. */
int refo_phase(void *hp, size_t t, size_t K, float expectIBDcM, float hist, float pErr, float pLimit,
               int doPrePhasing, int doRevPhasing,
               uint64_t *mat, uint64_t *pat, float *dos_mat, float *dos_pat,
               float *totalconf, size_t *ncallsites) {
    Handle *h = (Handle*)hp;
    VCFData &v = h->vd;
    size_t cap = capBytes(v.M);
    uint64_t *md = (uint64_t*)aligned_alloc(64, cap), *pd = (uint64_t*)aligned_alloc(64, cap);
    memset(md, 0, cap); memset(pd, 0, cap);
    BooleanVector pm(md, cap, 0), pp(pd, cap, 0);
    std::vector<float> dm, dp;
    {
        Target tg(pm, pp, dm, dp, t, v.targetIDs[t], v, v.Nrefhaps, h->ncorr(), K,
                  expectIBDcM, hist, pErr, pLimit, doPrePhasing, doRevPhasing, h->lastIter, false, false, false);
        tg.phase();
        *totalconf = tg.getTotalConfidence();
        *ncallsites = tg.getNCallSites();
    }
    memcpy(mat, md, cap); memcpy(pat, pd, cap);
    // a haploid target (Target.cpp:166-203) fills only the maternal dosages
    dm.resize(v.M, 0.0f);
    dp.resize(v.M, 0.0f);
    memcpy(dos_mat, dm.data(), v.M * sizeof(float));
    memcpy(dos_pat, dp.data(), v.M * sizeof(float));
    free(md); free(pd);
    return 0;
}

/* The reference's CPU phasing loop (PBWTPhaser.cpp:695-723): OpenMP
 * dynamic,1 over targets [t0, t1).  Outputs are indexed by t - t0. */
int refo_phase_range(void *hp, size_t t0, size_t t1, int nthreads, size_t K, float expectIBDcM,
                     float hist, float pErr, float pLimit, int doPrePhasing, int doRevPhasing,
                     uint64_t *mats, uint64_t *pats, float *dos_mats, float *dos_pats) {
    Handle *h = (Handle*)hp;
    size_t wM = capBytes(h->vd.M) / 8;
    omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t t = t0; t < t1; t++) {
        float tc; size_t nc;
        refo_phase(hp, t, K, expectIBDcM, hist, pErr, pLimit, doPrePhasing, doRevPhasing,
                   mats + (t - t0) * wM, pats + (t - t0) * wM,
                   dos_mats + (t - t0) * h->vd.M, dos_pats + (t - t0) * h->vd.M, &tc, &nc);
    }
    return 0;
}

/* PBWTImputer::prepareImputation (PBWTImputer.cpp:63-185) over phased target
 * haplotypes (2*ntarget x W(M) words, mat then pat per target). */
void *refo_imp_create(void *hp, const uint64_t *phased, unsigned nthreads, int setmaxerrors, int imputeCalls) {
    Handle *h = (Handle*)hp;
    VCFData &v = h->vd;
    ImpHandle *ih = new ImpHandle();
    ih->h = h;
    ih->statfile = "";
    size_t cap = capBytes(v.M);
    size_t nh = 2 * v.Ntarget;
    ih->pdata = (uint64_t*)aligned_alloc(64, nh * cap);
    memcpy(ih->pdata, phased, nh * cap);
    ih->phased.resize(nh);
    for (size_t i = 0; i < nh; i++) ih->phased[i].setData(ih->pdata + i * cap / 8, cap, v.M);
    ih->imp = new PBWTImputer(v, ih->statfile, nthreads, 1, setmaxerrors, imputeCalls != 0, false);
    std::vector<size_t> nsites = {0, v.Mref, 0};
    ih->imp->prepareImputation(ih->phased, nsites);
    return ih;
}

void refo_imp_destroy(void *ip) { delete (ImpHandle*)ip; }

/* New phased target haplotypes against the imputer's existing reference
 * PBWT: the match part of PBWTImputer::prepareImputation
 * (PBWTImputer.cpp:117-157) with the reference's own TargetImp, OpenMP
 * dynamic,1 over the haplotypes as there.  The PBWT is built once per
 * imputer; this times what each further set of targets costs. */
void refo_imp_retarget(void *ip, const uint64_t *phased, unsigned nthreads) {
    ImpHandle *ih = (ImpHandle*)ip;
    VCFData &v = ih->h->vd;
    PBWTImputer *imp = ih->imp;
    size_t cap = capBytes(v.M);
    memcpy(ih->pdata, phased, 2 * v.Ntarget * cap);
    std::vector<size_t> nsites = {0, v.Mref, 0};
    imp->targets.clear();
    imp->targets.reserve(imp->nTargetHap);
    for (size_t nhap = 0; nhap < imp->nTargetHap; nhap++)
        imp->targets.emplace_back(nhap, v, *imp->pbwt, ih->phased[v.getHaploidsTgtMap()[nhap]], imp->num_blocks,
                                  imp->setmaxerrors, imp->imputeCalls, imp->debug);
    omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t nhap = 0; nhap < imp->nTargetHap; nhap++) {
        imp->targets[nhap].calcSMMatches();
        imp->targets[nhap].prepareBlocks(nsites);
    }
}

/* haplotypes of the imputation PBWT (PBWTImputer.cpp:31-34: the panel's
 * haplotypes less one per haploid sample) and target haplotypes imputed */
size_t refo_imp_K(void *ip) { return ((ImpHandle*)ip)->imp->pbwt->K; }
size_t refo_imp_ntargethaps(void *ip) { return ((ImpHandle*)ip)->imp->nTargetHap; }

/* matches of the imputer's target haplotype `hap` (0..ntargethaps-1: the
 * haplotypes that exist, in the order of VCFData::getHaploidsTgtMap) */
size_t refo_imp_nmatches(void *ip, size_t hap) {
    ImpHandle *ih = (ImpHandle*)ip;
    return ih->imp->targets[hap].sm_matches.size();
}

/* set-maximal matches of one target haplotype as (start, end, refstart, refend) */
void refo_imp_matches(void *ip, size_t hap, int64_t *out) {
    ImpHandle *ih = (ImpHandle*)ip;
    const auto &mm = ih->imp->targets[hap].sm_matches;
    for (size_t i = 0; i < mm.size(); i++) {
        out[4*i] = mm[i].start; out[4*i+1] = mm[i].end;
        out[4*i+2] = mm[i].refstart; out[4*i+3] = mm[i].refend;
    }
}

/* reference PBWT of the imputer: compressed rows (M x 2*ceil(K/32) u32) and
 * the prefix arrays gAbsPerm ((M+1) x K int) */
void refo_imp_refpbwt(void *ip, uint32_t *compr, int32_t *absperm) {
    ImpHandle *ih = (ImpHandle*)ip;
    PBWT *p = ih->imp->pbwt;
    if (compr) memcpy(compr, p->comprPBWT, p->M * p->Kwords * sizeof(uint32_t));
    if (absperm)
        for (size_t m = 0; m <= p->M; m++)
            memcpy(absperm + m * p->K, p->gAbsPerm[m].data(), p->K * sizeof(int32_t));
}

/* one call of PBWTImputer::imputeBunch (PBWTImputer.cpp:187-204) for block 0:
 * bits: 2*ntarget x W(bsize) words (cleared here first); dos: 2*ntarget x bsize */
void refo_imp_bunch(void *ip, size_t bsize, unsigned nthreads, uint64_t *bits, float *dos) {
    ImpHandle *ih = (ImpHandle*)ip;
    VCFData &v = ih->h->vd;
    size_t nh = 2 * v.Ntarget;
    size_t cap = capBytes(bsize);
    memset(bits, 0, nh * cap);
    std::vector<BooleanVector> it(nh);
    for (size_t i = 0; i < nh; i++) it[i].setData(bits + i * cap / 8, cap, 0);
    std::vector<std::vector<float>> id(nh, std::vector<float>(bsize, 0.0f));
    ih->imp->setNumThreads(nthreads);
    ih->imp->imputeBunch(0, bsize, it, id);
    for (size_t i = 0; i < nh; i++) memcpy(dos + i * bsize, id[i].data(), bsize * sizeof(float));
}

// Qref haplotype vectors: the reference's own run-length coder (utils.h)
long refo_rle_encode(const uint64_t *src, size_t nwords, uint8_t *enc) {
    vector<char> out;
    if (!runlengthEncode(src, nwords, out)) return -1;
    memcpy(enc, out.data(), out.size());
    return (long)out.size();
}

void refo_rle_decode(const uint8_t *enc, size_t encsize, uint64_t *dest, size_t nwords) {
    vector<char> in((const char *)enc, (const char *)enc + encsize);
    vector<size_t> masked;
    vector<bool> maskedhap;
    size_t maskedalleles = 0;
    runlengthDecode(in, dest, nwords, masked, maskedhap, maskedalleles);
}

// runlengthDecode with masked reference samples (utils.h:194-, as
// qRefLoadNextVariant calls it for --excludeRefSamples): the kept haplotypes
// into nwords words; returns the masked variant alleles it counts.  The
// sequence must be well-formed (the reference exits on a truncated one).
size_t refo_rle_decode_masked(const uint8_t *enc, size_t encsize, uint64_t *dest, size_t nwords,
                              const uint64_t *masked, size_t nmasked, const uint8_t *maskedhap) {
    vector<char> in((const char *)enc, (const char *)enc + encsize);
    vector<size_t> m(masked, masked + nmasked);
    vector<bool> mh(nmasked);
    for (size_t i = 0; i < nmasked; i++) mh[i] = maskedhap[i] != 0;
    size_t maskedalleles = 0;
    runlengthDecode(in, dest, nwords, m, mh, maskedalleles);
    return maskedalleles;
}

// the haplotype section of a Qref file decoded variant by variant with the
// reference's runlengthDecode, as qRefLoadNextVariant does after its reads
// (VCFData.cpp:2378-2535; no masked samples); returns -2 for a short section
int refo_qref_decode(const uint8_t *sec, size_t nbytes, size_t Mref, size_t nwords, uint64_t *out) {
    vector<size_t> masked;
    vector<bool> maskedhap;
    size_t off = 0;
    for (size_t v = 0; v < Mref; v++) {
        if (off + 8 > nbytes) return -2;
        size_t encsize;
        memcpy(&encsize, sec + off, 8);
        off += 8;
        uint64_t *row = out + v * nwords;
        memset(row, 0, nwords * 8);
        if (encsize) {
            if (off + encsize > nbytes) return -2;
            vector<char> enc((const char *)sec + off, (const char *)sec + off + encsize);
            size_t maskedalleles = 0;
            runlengthDecode(enc, row, nwords, masked, maskedhap, maskedalleles);
            off += encsize;
        } else {
            if (off + nwords * 8 > nbytes) return -2;
            memcpy(row, sec + off, nwords * 8);
            off += nwords * 8;
        }
    }
    return 0;
}

} // extern "C"
