// C-ABI driver over the reference's own VCFData::writeVCFImputedBunch
// (VCFData.cpp:3068-3446), compiled unmodified from the reference tree into
// the test oracle (oracle/_ref/libeimp_refwriter.so).  Test infrastructure
// written for this project; nothing in the product path loads it.
//
// VCFData's constructor reads the input files, so the harness never runs it:
// refw_write_bunch takes zeroed storage for a VCFData, constructs exactly the
// members writeVCFImputedBunch reads (the chunk's site tables, the targets, the
// per-worker buffers and record queues that writeVCFImputedPrepare would make,
// the options), calls the writer for one bunch, and reads every record back
// from the queues: the FORMAT fields ADS, GT, DS, GP and the INFO fields
// RefPanelAF, AF, MAF, R2, AC, AN, TYPED as the writer set them, and the
// run-statistics counters (conflicts, the --improveCalls categories and
// totals).  A filtered record is a NULL in the queue.  One worker thread, so
// the counters (plain size_t in the reference) are not raced.
#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <queue>
#include <random>
#include <set>
#include <sstream>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

// the standard headers above come before the access override, which must
// only reach the reference's own class declarations
#define private public
#define protected public
#include "VCFData.h"
#undef private
#undef protected

#include "MyMalloc.h"
#include "StatusFile.h"

StatusFile StatusFile::instance;
MyMalloc MyMalloc::mm;

namespace {

size_t capBytes(size_t nbits) { return roundToMultiple(nbits, UNITWORDS * sizeof(uint64_t) * 8) / 8; }

template <typename T> void construct(T &member) { new (&member) T(); }
template <typename T> void destroy(T &member) { member.~T(); }

struct Storage {
    std::vector<void *> bufs;
    ~Storage() { for (void *p : bufs) std::free(p); }
    uint64_t *bits(size_t nbits, const uint64_t *src, size_t srcwords) {
        const size_t cap = capBytes(nbits);
        void *p = std::aligned_alloc(64, cap ? cap : 64);
        std::memset(p, 0, cap ? cap : 64);
        std::memcpy(p, src, std::min(cap, srcwords * 8));
        bufs.push_back(p);
        return static_cast<uint64_t *>(p);
    }
};

}  // namespace

extern "C" {

/* One bunch [mref_begin, mref_begin + nsites) of a chunk of Mref sites, with
 * N targets typed at the ascending sites typed[0..M-1]:
 *   bits   2N x wb words    imputed alleles of the bunch (imputedTargets)
 *   dos    2N x nsites      imputed dosages (imputedDosages; < 0 = conflict)
 *   phased 2N x wM words    phased haplotypes at the typed sites (phasedTargets)
 *   pdm, pdp N x M          phased dosages of mat/pat (phasedDosages 2i, 2i+1)
 *   gt     N x M            genotypes 0/1/2, 3 = missing (targets)
 *   af_full Mref            reference panel allele frequencies
 *   haploid N bytes or NULL (haploidsTgt)
 * Outputs per site s (nsites): written[s] (the record passed the filters),
 * and for written records: ads 2N x nsites, gtv 2N x nsites (BCF GT values),
 * ds N x nsites, gp 3N x nsites (GP0..2 of target i in rows 3i..3i+2),
 * info nsites x 4 (RefPanelAF, AF, MAF, R2), acan nsites x 2, typedflag.
 * ds/gp entries the writer leaves unset keep the value the caller put there.
 * counters: conflictcnt, improvecnt nochange, het2het, hom2hom, het2hom,
 * hom2het; totals: the five totalimprove sums in the same order. */
int refw_write_bunch(size_t N, size_t Mref, size_t mref_begin, size_t nsites, const uint64_t *bits, size_t wb,
                     const float *dos, const uint64_t *phased, size_t wM, const float *pdm, const float *pdp,
                     const uint8_t *gt, size_t M, const int64_t *typed, const float *af_full, const uint8_t *haploid,
                     int overwriteCalls, int improveCalls, float r2filter, float maffilter, uint8_t *written,
                     float *ads, int32_t *gtv, float *ds, float *gp, float *info, int32_t *acan, uint8_t *typedflag,
                     uint64_t *counters, double *totals) {
    if (mref_begin + nsites > Mref) return 1;
    void *mem = std::aligned_alloc(alignof(VCFData), (sizeof(VCFData) + alignof(VCFData) - 1) / alignof(VCFData) *
                                                         alignof(VCFData));
    std::memset(mem, 0, sizeof(VCFData));
    VCFData &v = *static_cast<VCFData *>(mem);
    Storage st;

    // chunk tables (one block covering the chunk, no region clipping)
    construct(v.site_offsets);
    v.site_offsets = {0, Mref};
    v.currChunkOffset = 0;
    construct(v.positionsFullRefRegion);
    v.positionsFullRefRegion.resize(Mref);
    for (size_t i = 0; i < Mref; i++) v.positionsFullRefRegion[i] = (int64_t)i + 1;
    v.startChunkBp = 0;
    v.endChunkBp = (int64_t)Mref + 1;
    v.excludeMultiAllRef = false;
    construct(v.variantIDsFullRefRegion);
    v.variantIDsFullRefRegion.assign(Mref, ".");
    construct(v.allelesFullRefRegion);
    v.allelesFullRefRegion.assign(2 * Mref, "A");
    construct(v.alleleFreqsFullRefRegion);
    v.alleleFreqsFullRefRegion.assign(af_full, af_full + Mref);
    construct(v.isImputed);
    v.isImputed.reset(Mref, 0);
    construct(v.ptgtIdx);
    v.ptgtIdx.reset(Mref, 0);
    for (size_t i = 0, k = 0; i < Mref; i++) {
        const bool ty = k < M && (size_t)typed[k] == i;
        v.isImputed.push_back(!ty);
        v.ptgtIdx.push_back(ty ? k : 0);
        if (ty) k++;
    }

    // targets
    v.Ntarget = N;
    construct(v.haploidsTgt);
    v.haploidsTgt.assign(N, false);
    if (haploid)
        for (size_t i = 0; i < N; i++) v.haploidsTgt[i] = haploid[i] != 0;
    construct(v.targets);
    v.targets.resize(N);
    for (size_t t = 0; t < N; t++) {
        v.targets[t].reserve(M);
        for (size_t m = 0; m < M; m++) v.targets[t].push_back((Genotype)gt[t * M + m]);
    }

    // options
    v.num_workers = 1;
    v.imp_hdr = nullptr;
    v.writeADosage = true;
    v.writeGDosage = ds != nullptr;
    v.writeProbs = gp != nullptr;
    v.overwriteCalls = overwriteCalls != 0;
    v.improveCalls = improveCalls != 0;
    v.impR2filter = r2filter;
    v.impMAFfilter = maffilter;

    // per-worker buffers and queues (writeVCFImputedPrepare, VCFData.cpp:2967-3066)
    construct(v.ads_vec);
    construct(v.ds_vec);
    construct(v.gp_vec);
    construct(v.tgt_gt_vec);
    construct(v.mtgt_gt_vec);
    construct(v.recqs);
    v.ads_vec.assign(1, std::vector<float>(2 * N));
    v.ds_vec.assign(1, std::vector<float>(N));
    v.gp_vec.assign(1, std::vector<float>(3 * N));
    std::vector<int32_t> gtbuf(2 * N);
    v.tgt_gt_vec.assign(1, gtbuf.data());
    v.recqs.resize(1);
    v.recqs[0].resize(1);

    // results of phasing and imputation of the bunch
    std::vector<BooleanVector> imputedTargets(2 * N), phasedTargets(2 * N);
    std::vector<std::vector<float>> imputedDosages(2 * N), phasedDosages(2 * N);
    for (size_t h = 0; h < 2 * N; h++) {
        imputedTargets[h].setData(st.bits(nsites, bits + h * wb, wb), capBytes(nsites), nsites);
        phasedTargets[h].setData(st.bits(M, phased + h * wM, wM), capBytes(M), M);
        imputedDosages[h].assign(dos + h * nsites, dos + (h + 1) * nsites);
        const float *pd = (h & 1) ? pdp : pdm;
        phasedDosages[h].assign(pd + (h / 2) * M, pd + (h / 2 + 1) * M);
    }

    // the stale-value behaviour of the per-worker DS/GP buffers is kept: the
    // buffers start as the caller's first site column
    if (ds)
        for (size_t i = 0; i < N; i++) v.ds_vec[0][i] = ds[i * nsites];
    if (gp)
        for (size_t i = 0; i < 3 * N; i++) v.gp_vec[0][i] = gp[i * nsites];

    v.writeVCFImputedBunch(0, mref_begin, nsites, imputedTargets, imputedDosages, phasedTargets, phasedDosages);

    int rc = 0;
    for (size_t s = 0; s < nsites; s++) {
        bcf1_t *rec = nullptr;
        if (!v.recqs[0][0].try_pop(rec)) { rc = 2; break; }
        written[s] = rec != nullptr;
        if (!rec) continue;
        const auto &A = rec->fmt_f["ADS"];
        const auto &G = rec->fmt_i["GT"];
        for (size_t h = 0; h < 2 * N; h++) {
            ads[h * nsites + s] = A[h];
            gtv[h * nsites + s] = G[h];
        }
        if (ds) {
            const auto &D = rec->fmt_f["DS"];
            for (size_t i = 0; i < N; i++) ds[i * nsites + s] = D[i];
        }
        if (gp) {
            const auto &P = rec->fmt_f["GP"];
            for (size_t i = 0; i < 3 * N; i++) gp[i * nsites + s] = P[i];
        }
        info[4 * s + 0] = rec->info_f["RefPanelAF"][0];
        info[4 * s + 1] = rec->info_f["AF"][0];
        info[4 * s + 2] = rec->info_f["MAF"][0];
        info[4 * s + 3] = rec->info_f["R2"][0];
        acan[2 * s + 0] = rec->info_i["AC"][0];
        acan[2 * s + 1] = rec->info_i["AN"][0];
        typedflag[s] = rec->info_flag.count("TYPED") ? 1 : 0;
        delete rec;
    }
    counters[0] = v.conflictcnt;
    counters[1] = v.improvecntnochange;
    counters[2] = v.improvecnthet2het;
    counters[3] = v.improvecnthom2hom;
    counters[4] = v.improvecnthet2hom;
    counters[5] = v.improvecnthom2het;
    totals[0] = v.totalimprovenochange;
    totals[1] = v.totalimprovehet2het;
    totals[2] = v.totalimprovehom2hom;
    totals[3] = v.totalimprovehet2hom;
    totals[4] = v.totalimprovehom2het;
    // only the members constructed above are destroyed (VCFData's own
    // destructor would free buffers and headers the harness never made)
    destroy(v.site_offsets);
    destroy(v.positionsFullRefRegion);
    destroy(v.variantIDsFullRefRegion);
    destroy(v.allelesFullRefRegion);
    destroy(v.alleleFreqsFullRefRegion);
    destroy(v.isImputed);
    destroy(v.ptgtIdx);
    destroy(v.haploidsTgt);
    destroy(v.targets);
    destroy(v.ads_vec);
    destroy(v.ds_vec);
    destroy(v.gp_vec);
    destroy(v.tgt_gt_vec);
    destroy(v.mtgt_gt_vec);
    destroy(v.recqs);
    std::free(mem);
    return rc;
}

}  // extern "C"
