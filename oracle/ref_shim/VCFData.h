/*
 * Stand-in for the reference's VCFData class, used ONLY to build the
 * reference's own hot-path sources (Target, PBWT, Beam*, HaplotypePath,
 * TargetImp, PBWTImputer, ...) into the test oracle under oracle/_ref/.
 *
 * This header is test infrastructure written for this project.  It offers
 * exactly the accessors the hot path calls (VCFData.h:80-115 of the
 * reference) backed by plain members that the oracle driver fills from
 * in-memory arrays; it reads no VCF/BCF/Qref file and needs no htslib, TBB or
 * Boost.  Layouts follow the reference:
 *   reference       -- typed sites, one BooleanVector per haplotype (VCFData.h:199)
 *   referenceT      -- typed sites, one BooleanVector per site    (VCFData.h:201)
 *   referenceFullT  -- all panel sites, one BooleanVector per site (VCFData.h:211)
 *   targets         -- GenotypeVector per target (VCFData.h:216)
 */
#ifndef VCFDATA_H_
#define VCFDATA_H_

#include <string>
#include <vector>

#include "Datatypes.h"
#include "RingBuffer.h"
#include "MyMalloc.h"

using namespace std;

class VCFData {
public:
    VCFData() : cMs(16, 0), Nrefhaps(0), Ntarget(0), M(0), Mref(0) {}

    const vector<BooleanVector> &getReference_const() const { return reference; }
    const RingBuffer<BooleanVector> &getReferenceT_const() const { return referenceT; }
    vector<BooleanVector> &getReference() { return reference; }
    RingBuffer<BooleanVector> &getReferenceT() { return referenceT; }
    const vector<BooleanVector> &getReferenceFullT() const { return referenceFullT; }
    const vector<GenotypeVector> &getTargets() const { return targets; }
    const vector<RingBuffer<size_t>> &getTgtMissPos() const { return tgtmiss; }
    const vector<RingBufferBool> &getTgtInPhases() const { return tgtinphase; }
    const RingBuffer<fp_type> &getCMPos() const { return cMs; }
    const vector<string> &getTargetIDs() const { return targetIDs; }

    // in phasing iterations after the first the panel holds the reference
    // haplotypes followed by the phased targets: getNReferenceHaps is the
    // reference part, getNReferenceHapsMax all of it (VCFData.h of the reference)
    size_t getNReferenceHaps() const { return NrefhapsOrig ? NrefhapsOrig : Nrefhaps; }
    size_t getNReferenceHapsMax() const { return Nrefhaps; }
    size_t getNTarget() const { return Ntarget; }
    size_t getNSNPs() const { return M; }
    size_t getNSNPsFullRef() const { return Mref; }
    size_t getSNPIndexToFullRef(size_t tgtsnpindex) const { return indexToRefFull[tgtsnpindex]; }
    float getAlleleFreqFullRefRegion(size_t i) const { return alleleFreqsFullRefRegion[i]; }
    float getAlleleFreqCommon(size_t i) const { return alleleFreqsCommon[i]; }
    const vector<bool> &getHaploidsRef() const { return haploidsRef; }
    const vector<bool> &getHaploidsTgt() const { return haploidsTgt; }
    const vector<size_t> &getHaploidsRefMap() const { return haploidsRefMap; }
    const vector<size_t> &getHaploidsTgtMap() const { return haploidsTgtMap; }
    size_t getNHaploidsRef() const { return nHaploidsRef; }
    size_t getNHaploidsTgt() const { return nHaploidsTgt; }
    Haplotype getStartPhase(size_t targetidx) const { return toHap(chunkStartPhase[targetidx]); }

    // plain storage, filled by the oracle driver
    size_t NrefhapsOrig = 0;
    vector<BooleanVector> reference;
    RingBuffer<BooleanVector> referenceT;
    vector<BooleanVector> referenceFullT;
    vector<GenotypeVector> targets;
    vector<RingBuffer<size_t>> tgtmiss;
    vector<RingBufferBool> tgtinphase;
    RingBuffer<fp_type> cMs;
    vector<string> targetIDs;
    size_t Nrefhaps;
    size_t Ntarget;
    size_t M;
    size_t Mref;
    vector<size_t> indexToRefFull;
    vector<float> alleleFreqsFullRefRegion;
    vector<float> alleleFreqsCommon;
    vector<bool> haploidsRef, haploidsTgt;
    vector<size_t> haploidsRefMap, haploidsTgtMap;
    size_t nHaploidsRef = 0, nHaploidsTgt = 0;
    vector<bool> chunkStartPhase;
};

#endif /* VCFDATA_H_ */
