// Allocation-free best-haplotype selection.
//
// Some callers cannot let a library allocate device memory: a host framework
// that owns the whole device budget through its own pool (a cudaMalloc behind
// its back fragments or exhausts that budget), or a serving process that
// allocates everything at start-up and forbids allocation on its request path.
// For them, eimp_besthaps_noalloc runs the best-haplotype selection (the
// Hamming counts of every target against every reference haplotype, then the
// K smallest) on buffers the caller provides, with the per-haplotype error
// counts kept in the fixed device array below instead of an allocated scratch
// buffer.  It needs no context and calls no cudaMalloc/cudaFree.
//
// The array is a module global: every GPU that loads this library holds
// EIMP_BESTHAPS_NOALLOC_MAX * 4 bytes (16 MiB) of it until the process exits,
// and all calls on one device share it.
#include <cstdio>
#include <mutex>

#include "common.cuh"
#include "kernels.h"
#include "../../include/eimp_gpu.h"

namespace {

// error counts of the last call: one uint32 per (target, reference haplotype);
// every call overwrites the entries it reads, so nothing needs clearing
__device__ __align__(256) uint32_t g_besthaps_nerr[EIMP_BESTHAPS_NOALLOC_MAX];

constexpr int kMaxDevices = 64;
uint32_t *g_nerr_addr[kMaxDevices] = {nullptr};
std::mutex g_nerr_mutex;

// device address of the array on the current device (set-up once per device;
// the address stays valid for the life of the device's primary context, so a
// cudaDeviceReset after the first call is not supported)
int nerr_address(uint32_t **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return EIMP_E_CUDA;
    std::lock_guard<std::mutex> lk(g_nerr_mutex);
    if (!g_nerr_addr[dev]) {
        void *p = nullptr;
        // host code only knows a stand-in for the array's name; the device
        // address has to be looked up with the device current
        if (cudaGetSymbolAddress(&p, g_besthaps_nerr) != cudaSuccess || !p) return EIMP_E_CUDA;
        g_nerr_addr[dev] = static_cast<uint32_t *>(p);
    }
    *out = g_nerr_addr[dev];
    return EIMP_OK;
}

}  // namespace

extern "C" int eimp_besthaps_noalloc(void *stream, size_t ntgt, size_t M, const uint8_t *d_gt,
                                     const uint64_t *d_hapmajor, size_t nhaps, size_t K, int32_t *d_besthaps,
                                     uint64_t *d_flags) {
    if (!ntgt || !M || !nhaps || !K || !d_gt || !d_hapmajor || !d_besthaps || !d_flags) return EIMP_E_ARG;
    if (ntgt > (size_t)EIMP_BESTHAPS_NOALLOC_MAX / nhaps) return EIMP_E_CAPACITY;
    if (M > (size_t)INT32_MAX || nhaps > (size_t)INT32_MAX) return EIMP_E_ARG;
    // the kernel keeps the target's two genotype bit vectors in shared memory
    // (16 * W(M) bytes per CTA): longer targets do not fit a CTA
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return EIMP_E_CUDA;
    if ((size_t)16 * eimp_W(M) > (size_t)optin) return EIMP_E_CAPACITY;
    uint32_t *nerr = nullptr;
    if (int r = nerr_address(&nerr)) return r;
    const size_t Kc = K < nhaps ? K : nhaps;
    cudaError_t e = eimp::launch_besthaps(d_gt, (int)ntgt, (int)M, d_hapmajor, (int)nhaps, (int)eimp_W(M), (int)Kc,
                                          nerr, d_besthaps, d_flags, (int)eimp_W(nhaps), -1, nullptr,
                                          static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? EIMP_OK : EIMP_E_CUDA;
}
