// Shared device helpers for the EagleImp B200 kernels.
//
// Bit layouts follow the reference: bit vectors are uint64 words, least
// significant bit first, rows padded to 512-bit units (Datatypes.h:70).
// Compressed PBWT rows are 2*ceil(K/32) uint32: pairs of [32 data bits in
// prefix order, cumulative zeros through this word], the tail word padded with
// ones (PBWT.cpp:236-267).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#define EIMP_HD __host__ __device__ __forceinline__
#define EIMP_D __device__ __forceinline__

EIMP_HD size_t eimp_W(size_t nbits) { return ((nbits + 511) / 512) * 8; }
EIMP_HD size_t eimp_kw(size_t K) { return 2 * ((K + 31) / 32); }

EIMP_D int bit_at(const uint64_t *v, size_t i) { return (int)((v[i >> 6] >> (i & 63)) & 1ull); }

// PBWT::decodeRelPerm (PBWT.cpp:367-382): position of element 'from' after
// the stable 0/1 partition of this row
EIMP_D int pbwt_rank(const uint32_t *row, int cnt0, int from) {
    const uint2 pr = reinterpret_cast<const uint2 *>(row)[from >> 5];   // [data, zeros] pair
    uint32_t off = pr.y;
    uint32_t field = pr.x;
    uint32_t mask = 1u << (from & 31);
    uint32_t bit = field & mask;
    field |= mask - 1u;
    uint32_t fcnt0 = off - (uint32_t)__popc(~field);
    return bit ? cnt0 + (from - (int)fcnt0) : (int)fcnt0;
}

// PBWT::mapInterval (PBWT.cpp:304-365).  Empty interval: l > r (0, -1).
EIMP_D void pbwt_map(const uint32_t *row, int cnt0, int l, int r, int &l0, int &r0, int &l1, int &r1) {
    l0 = 0; r0 = -1; l1 = 0; r1 = -1;
    if (l > r) return;
    if (l == r) {
        int i = pbwt_rank(row, cnt0, l);
        if (i < cnt0) { l0 = i; r0 = i; } else { l1 = i; r1 = i; }
        return;
    }
    int a0 = pbwt_rank(row, cnt0, l);
    int a1 = l - a0 + cnt0;
    if (a0 >= cnt0) { int t = a0; a0 = a1; a1 = t; }
    int b0 = pbwt_rank(row, cnt0, r);
    int b1 = r - b0 + cnt0 - 1;
    if (b0 >= cnt0) { int t = b0; b0 = b1; b1 = t; }
    l0 = a0; r0 = b0; l1 = a1; r1 = b1;
}

// error flags a kernel may raise (ORed into a device status word)
enum : uint32_t {
    EIMP_ERR_MATCH_OVERFLOW = 1u << 0,   // set-maximal match buffer full
    EIMP_ERR_NODE_OVERFLOW  = 1u << 1,   // match-tree node pool full
    EIMP_ERR_STACK_OVERFLOW = 1u << 2,   // match-tree traversal stack full
    EIMP_ERR_BEAM_EMPTY     = 1u << 3,   // "Beam is empty. No paths left." (Beam.cpp:466-470)
    EIMP_ERR_BEAM_CAPACITY  = 1u << 4,   // beam/happath pool exhausted
    EIMP_ERR_ROWS_OVERFLOW  = 1u << 5,   // condensed reference rows exceed the buffer
    EIMP_ERR_QREF_TRUNCATED = 1u << 6,   // "Truncated runlength sequence!" (utils.h:222-240)
    EIMP_ERR_HAPLOID_HET    = 1u << 7,   // "Found heterozygous genotype in haploid target." (Target.cpp:196-199)
};
