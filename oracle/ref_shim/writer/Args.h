/*
 * Stand-in for the reference's Args class (Args.h, which needs Boost's
 * program_options), used ONLY to compile the reference's VCFData.cpp into the
 * writer harness of the test oracle.  It holds the option fields VCFData.cpp
 * reads, with the reference's names and types, and no parser: the harness
 * never runs VCFData's constructor.
 */
#ifndef ARGS_H_
#define ARGS_H_

#include <cstdint>
#include <string>
#include <vector>

#include "Datatypes.h"

using namespace std;

class Args {
public:
    unsigned num_threads = 1;
    string outPrefix, genMapFile, ref, vcfTarget, vcfExclude, sampleList, writeMode;
    bool isQRef = false, createQuickRef = false, impMissing = false, allowRefAltSwap = false,
         allowStrandFlip = false, excludeMultiAllRef = false, outputUnphased = false, skipImputation = false,
         noMissingIDs = false, skipPhasing = false, writeADosage = false, writeGDosage = false, writeProb = false,
         overwriteCalls = false, improveCalls = false, skipHeader = false, deterministic = false, debug = false,
         yaml = false;
    float impR2filter = 0, impMAFfilter = 0;
    int64_t bpStart = 0, bpEnd = 0, bpFlanking = 0;
    uint64_t maxChunkMemory = 0, chunkFlankSize = 0;
    size_t K = 0, ibunchsize = 0, impR = 0;
    uint32_t iters = 1;
    unsigned num_files = 1;
};

#endif
