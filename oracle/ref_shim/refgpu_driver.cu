// C ABI over the reference's own GPU engine (GPUEngine.cu / GPUKernels.cu,
// compiled unmodified from the reference tree): GPUEngine::initialize /
// getBlockSize / runCrefPBWTKernel / free (GPUEngine.h:41-99).  TEST
// INFRASTRUCTURE: the reference's GPU form of the condensed reference and
// compressed PBWTs, run beside this project's drop-in on the same inputs for
// parity and timing.  Errors (the engine throws thrust::system_error) become
// a nonzero return code and a message.
#include <cstring>
#include <string>
#include <vector>

#include "GPUEngine.h"

static std::string g_err;

extern "C" {

const char *refgpu_last_error() { return g_err.c_str(); }

void *refgpu_create(int index) { return new GPUEngine(index); }

int refgpu_initialize(void *h, size_t K, size_t Kwords, size_t M, size_t Nrefhapscorr, size_t NrefhapsAD,
                      size_t refTCapacity, const uint64_t *refTData) {
    try {
        static_cast<GPUEngine *>(h)->initialize(K, Kwords, M, Nrefhapscorr, NrefhapsAD, refTCapacity, refTData);
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
    return 0;
}

size_t refgpu_block_size(void *h) { return static_cast<GPUEngine *>(h)->getBlockSize(); }

// count0s[t] receives crefTOffsets[t+1] - crefTOffsets[t] ints
int refgpu_run(void *h, size_t ntgt, const uint64_t *const *tgtData, const uint64_t *const *splitData,
               const uint64_t *const *besthapData, const uint32_t *crefTOffsets, uint32_t *const *cPBWT,
               int *const *count0s) {
    std::vector<const data_type *> tgt(tgtData, tgtData + ntgt), spl(splitData, splitData + ntgt),
        bh(besthapData, besthapData + ntgt);
    std::vector<uint32_t> off(crefTOffsets, crefTOffsets + ntgt + 1);
    std::vector<uint32_t *> out(cPBWT, cPBWT + ntgt);
    std::vector<std::vector<int>> c0(ntgt);
    std::vector<std::vector<int> *> c0p(ntgt);
    for (size_t t = 0; t < ntgt; t++) {
        c0[t].resize(off[t + 1] - off[t]);
        c0p[t] = &c0[t];
    }
    try {
        static_cast<GPUEngine *>(h)->runCrefPBWTKernel(tgt, spl, bh, off, out, c0p);
    } catch (const std::exception &e) {
        g_err = e.what();
        return -1;
    }
    for (size_t t = 0; t < ntgt; t++) std::memcpy(count0s[t], c0[t].data(), c0[t].size() * sizeof(int));
    return 0;
}

void refgpu_destroy(void *h) {
    GPUEngine *e = static_cast<GPUEngine *>(h);
    e->free();
    delete e;
}

}  // extern "C"
