// Qref reference panel: decoding of the haplotype section on the device
// (sm_100a).
//
//  qref_decode_kernel -- VCFData::qRefLoadNextVariant (VCFData.cpp:2378-2535)
//                        with runlengthDecode (utils.h:194-), no masked
//                        samples: every variant's haplotype vector, stored
//                        raw or run-length coded (qref_spec.md section I),
//                        into its row of the site-major panel
//                        (referenceFullT).
//  qref_mask_kernel   -- the same with masked reference samples
//                        (--excludeRefSamples, VCFData.cpp:2405-2523): the
//                        decoded row with the masked samples' bit pairs
//                        removed, and the panel allele frequency corrected
//                        for the masked variant alleles.
//
// The host copies the section as it lies in the file (one transfer) and the
// byte offset of every variant's <encsize> field (a walk over the size
// fields, qref_index on the host); one warp then decodes one variant.  A raw
// vector is copied with 32-bit loads realigned by funnel shifts (the section
// interleaves 8-byte sizes with odd-length codes, so a vector can start at
// any byte).  A run-length code is read 32 bytes at a time: a ballot of the
// bytes' high bits and a few bit operations on it give the bytes that start
// a run length (a length is one byte, or two when the first has its high bit
// set);
// a warp scan of the lengths gives every run's first bit; runs alternate
// 0/1 starting with 0, and the lanes holding runs of ones set them in the
// zeroed row.  HBM-bound: each variant reads its code and writes its row.
#include "common.cuh"
#include "kernels.h"

namespace eimp {

__device__ __forceinline__ void set_ones(uint64_t *row, uint64_t a, uint64_t b) {   // bits [a, b), b > a
    const uint64_t wa = a >> 6, wb = (b - 1) >> 6;
    const int la = (int)(a & 63), lb = (int)((b - 1) & 63);
    if (wa == wb) {
        const uint64_t m = (lb == 63 ? ~0ull : ((1ull << (lb + 1)) - 1ull)) & (~0ull << la);
        atomicOr(reinterpret_cast<unsigned long long *>(row + wa), m);
        return;
    }
    atomicOr(reinterpret_cast<unsigned long long *>(row + wa), ~0ull << la);
    for (uint64_t w = wa + 1; w < wb; w++) row[w] = ~0ull;   // words inside the run belong to it alone
    atomicOr(reinterpret_cast<unsigned long long *>(row + wb), lb == 63 ? ~0ull : ((1ull << (lb + 1)) - 1ull));
}

__global__ void __launch_bounds__(128) qref_decode_kernel(const uint8_t *__restrict__ sec,
                                                          const int64_t *__restrict__ offs, int Mref, int nwords,
                                                          uint64_t *__restrict__ out, size_t ldw,
                                                          uint32_t *__restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (v >= Mref) return;
    const uint8_t *p = sec + offs[v];
    uint64_t encsize = 0;
    if (lane < 8) encsize = (uint64_t)p[lane] << (8 * lane);
    for (int o = 4; o; o >>= 1) encsize |= __shfl_xor_sync(0xffffffffu, encsize, o);
    encsize = __shfl_sync(0xffffffffu, encsize, 0);
    const uint8_t *enc = p + 8;
    uint64_t *row = out + (size_t)v * ldw;
    if (encsize == 0) {   // the raw vector (VCFData.cpp:2434-2446)
        const size_t mis = reinterpret_cast<uintptr_t>(enc) & 3u;
        const uint32_t *src = reinterpret_cast<const uint32_t *>(enc - mis);
        uint32_t *dst = reinterpret_cast<uint32_t *>(row);
        const unsigned sh = (unsigned)mis * 8u;
        for (int k = lane; k < 2 * nwords; k += 32)
            dst[k] = sh ? __funnelshift_r(src[k], src[k + 1], sh) : src[k];
        return;
    }
    for (int k = lane; k < nwords; k += 32) row[k] = 0ull;
    __syncwarp();
    const uint64_t nbits = (uint64_t)nwords * 64;
    int carry = 0;            // the chunk starts with the second byte of a run length
    unsigned long long runs = 0, pos = 0, last_start = 0;
    unsigned bnext = lane < encsize ? enc[lane] : 0u;   // the chunks are loaded one ahead
    for (uint64_t base = 0; base < encsize; base += 32) {
        const uint64_t i = base + lane;
        const bool in = i < encsize;
        const unsigned b = bnext;
        bnext = i + 32 < encsize ? enc[i + 32] : 0u;
        const unsigned hi = __ballot_sync(0xffffffffu, in && (b & 0x80u));
        const int nvalid = (int)min((uint64_t)32, encsize - base);
        // the bytes that start a run length, bit-parallel: inside every run of
        // high-bit bytes that begins at a start p, the bytes p+1, p+3, ... (up
        // to the byte after the run) are second bytes.  Adding a run's first
        // bit to the run carries through it; the carried bits at odd distance
        // from p are those second bytes.
        const uint64_t vmask = (1ull << nvalid) - 1ull;
        uint64_t H = (uint64_t)hi & vmask;
        if (carry) H &= ~1ull;   // byte 0 is the second byte of the previous chunk's last length
        const uint64_t P = H & ~(H << 1);
        const uint64_t EV = 0x5555555555555555ull, OD = 0xAAAAAAAAAAAAAAAAull;
        const uint64_t pe = P & EV, po = P & OD;
        const uint64_t cont = (((H + pe) ^ H ^ pe) & OD) | (((H + po) ^ H ^ po) & EV);
        uint64_t S = vmask & ~cont;
        if (carry) S &= ~1ull;
        const unsigned sm = (unsigned)S;
        const int ncarry = (int)((cont >> nvalid) & 1ull);
        const bool start = (sm >> lane) & 1u;
        unsigned nb = __shfl_down_sync(0xffffffffu, b, 1);
        const unsigned nb0 = __shfl_sync(0xffffffffu, bnext, 0);   // the next chunk's first byte
        if (lane == 31) nb = nb0;
        const unsigned len = start ? ((b & 0x80u) ? ((nb & 0xffu) << 7) | (b & 0x7fu) : b) : 0u;
        unsigned incl = len;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        const unsigned total = __shfl_sync(0xffffffffu, incl, 31);
        const unsigned long long rs = pos + (incl - len);
        const unsigned long long ridx = runs + __popc(sm & ((1u << lane) - 1u));
        if (start && (ridx & 1ull) && len && rs < nbits)   // a run of ones
            set_ones(row, rs, min(rs + len, (unsigned long long)nbits));
        const unsigned lastlane = sm ? 31 - __clz(sm) : 0;
        const unsigned long long ls = __shfl_sync(0xffffffffu, rs, lastlane);
        if (sm) last_start = ls;
        pos += total;
        runs += __popc(sm);
        carry = ncarry;
    }
    // utils.h:222-240: a run length cut after its first byte, or runs that end
    // inside a word the reference still decodes, are a truncated sequence
    const bool cut = carry != 0;
    const bool midword = (pos & 63ull) && (pos >> 6) <= max((unsigned long long)nwords - 1, last_start >> 6);
    if (lane == 0 && (cut || midword)) atomicOr(status, EIMP_ERR_QREF_TRUNCATED);
}

// 32 bits -> the even bits of a 64-bit word
__device__ __forceinline__ uint64_t spread_even(uint32_t b) {
    uint64_t x = b;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

// One warp per variant: rows (the decoded rows, 2 bits per sample) -> out
// (the kept samples' pairs in order, then zeros, nwout words).  The masked
// variant alleles are counted by the rule of the variant's storage: a raw
// vector counts a masked sample once if either bit is set and once more for
// a diploid 11 (VCFData.cpp:2471-2477); a run-length code counts each set
// bit of a diploid sample and, for a haploid one, the second bit after a set
// first bit (utils.h runlengthDecode, the masked-haplotype loop).  af[v] <-
// (float(an_before) * af - masked) / float(an_after) in float arithmetic
// (VCFData.cpp:2429-2434, 2517-2521).
__global__ void __launch_bounds__(128) qref_mask_kernel(
    const uint8_t *__restrict__ sec, const int64_t *__restrict__ offs, int nvar, const uint64_t *__restrict__ rows,
    size_t ldr, const int32_t *__restrict__ kept, int nkept, int nwout, const int64_t *__restrict__ masked,
    int nmasked, const uint8_t *__restrict__ masked_hap, float an_before, float an_after, float *__restrict__ af,
    uint64_t *__restrict__ out, size_t ldo) {
    const int lane = threadIdx.x & 31;
    const int v = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (v >= nvar) return;
    const uint8_t *p = sec + offs[v];
    uint64_t encsize = 0;
    if (lane < 8) encsize = (uint64_t)p[lane] << (8 * lane);
    for (int o = 4; o; o >>= 1) encsize |= __shfl_xor_sync(0xffffffffu, encsize, o);
    const bool raw = __shfl_sync(0xffffffffu, encsize, 0) == 0;
    const uint64_t *row = rows + (size_t)v * ldr;
    int cnt = 0;
    for (int i = lane; i < nmasked; i += 32) {
        const int64_t sm = masked[i];
        const int pair = (int)((row[sm >> 5] >> ((sm & 31) * 2)) & 3ull);
        const bool hap = masked_hap[i] != 0;
        cnt += raw ? (pair != 0) + (pair == 3 && !hap) : (hap ? (pair == 3) : __popc(pair));
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    uint64_t *orow = out + (size_t)v * ldo;
    for (int w = 0; w < nwout; w++) {
        const int k = w * 32 + lane;
        int pair = 0;
        if (k < nkept) {
            const int sk = kept[k];
            pair = (int)((row[sk >> 5] >> ((sk & 31) * 2)) & 3ull);
        }
        const unsigned b0 = __ballot_sync(0xffffffffu, pair & 1), b1 = __ballot_sync(0xffffffffu, pair & 2);
        if (lane == 0) orow[w] = spread_even(b0) | (spread_even(b1) << 1);
    }
    if (lane == 0) af[v] = __fdiv_rn(__fsub_rn(__fmul_rn(an_before, af[v]), (float)cnt), an_after);
}

cudaError_t launch_qref_mask(const uint8_t *sec, const int64_t *offs, int nvar, const uint64_t *rows, size_t ldr,
                             const int32_t *kept, int nkept, int nwout, const int64_t *masked, int nmasked,
                             const uint8_t *masked_hap, float an_before, float an_after, float *af, uint64_t *out,
                             size_t ldo, cudaStream_t st) {
    if (nvar <= 0) return cudaSuccess;
    qref_mask_kernel<<<(nvar + 3) / 4, 128, 0, st>>>(sec, offs, nvar, rows, ldr, kept, nkept, nwout, masked, nmasked,
                                                     masked_hap, an_before, an_after, af, out, ldo);
    return cudaGetLastError();
}

cudaError_t launch_qref_decode(const uint8_t *sec, const int64_t *offs, int Mref, int nwords, uint64_t *out,
                               size_t ldw, uint32_t *status, cudaStream_t st) {
    if (Mref <= 0) return cudaSuccess;
    qref_decode_kernel<<<(Mref + 3) / 4, 128, 0, st>>>(sec, offs, Mref, nwords, out, ldw, status);
    return cudaGetLastError();
}

}  // namespace eimp
