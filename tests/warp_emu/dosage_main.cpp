// Runs the dosage kernel (generated host copy of the dosage section of
// eimp_b200/csrc/imp_kernels.cu) one warp at a time under the warp emulator.
//
//   dosage_emu <dir>
//
// <dir> holds the inputs as raw little-endian arrays in the layout of the
// device buffers: params_i.bin (nhaps, cap, K, wMref, M, wM, nrefhaps_total,
// mref_begin, nsites, imputeCalls, Mref[, nrows, maps]), matches.bin (nhaps x cap int4),
// nmatch.bin (nhaps i32), absperm.bin ((M+1) x K i32), hapfull.bin (K x wMref
// u64), typed.bin (M i64), af.bin (Mref f32), phased.bin (nhaps x wM u64),
// gt.bin (nhaps/2 x M u8).  The segment map and the per-site pairs come from
// the segment-map kernel, run site by site.  Outputs: o_dos.bin (nhaps x
// nsites f32), o_bits.bin (nhaps x ceil(nsites/64) u64), o_segm.bin,
// o_sinfo.bin.  With maps set, the matches, phased rows and outputs have
// nrows rows (the target haplotypes), of which the nhaps listed in
// hapmap.bin are imputed, and refmap.bin gives the panel column of each
// haplotype of the reduced reference (hapfull.bin then has the panel's
// columns).  Every input is its own allocation so the address sanitizer
// sees reads past it.
// Exit status 3: a divergent warp collective was seen.
#include "dosage_emu.cpp"

#include <string>
#include <thread>
#include <vector>

thread_local dim3 threadIdx, blockIdx, blockDim;
thread_local EmuWarp *emu_warp;
thread_local EmuBarrier *emu_block;
thread_local uint8_t *emu_smem_ptr;
std::atomic<int> emu_divergence{0};

template <class T> static std::vector<T> rd(const std::string &d, const char *name) {
    const std::string p = d + "/" + name;
    FILE *f = fopen(p.c_str(), "rb");
    if (!f) { perror(p.c_str()); exit(1); }
    fseek(f, 0, SEEK_END);
    const long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<T> v(n / sizeof(T));
    if (fread(v.data(), 1, n, f) != (size_t)n) exit(2);
    fclose(f);
    return v;
}
template <class T> static void wr(const std::string &d, const char *name, const std::vector<T> &v) {
    const std::string p = d + "/" + name;
    FILE *f = fopen(p.c_str(), "wb");
    if (!f) { perror(p.c_str()); exit(1); }
    fwrite(v.data(), sizeof(T), v.size(), f);
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc < 2) { fprintf(stderr, "usage: %s <dir>\n", argv[0]); return 1; }
    const std::string d = argv[1];
    const auto pi = rd<int32_t>(d, "params_i.bin");
    const int nhaps = pi[0], cap = pi[1], K = pi[2], wMref = pi[3], M = pi[4], wM = pi[5], ntot = pi[6];
    const int mref_begin = pi[7], nsites = pi[8], impcalls = pi[9], Mref = pi[10];
    // optional: nrows target haplotype rows of which the nhaps in hapmap.bin
    // are imputed, and refmap.bin, the panel column of each of the K
    // haplotypes of the reduced reference (haploid samples)
    const int nrows = pi.size() > 11 ? pi[11] : nhaps;
    const bool maps = pi.size() > 12 && pi[12];
    const std::vector<int32_t> hapmap = maps ? rd<int32_t>(d, "hapmap.bin") : std::vector<int32_t>();
    const std::vector<int32_t> refmap = maps ? rd<int32_t>(d, "refmap.bin") : std::vector<int32_t>();
    const auto matches = rd<int4>(d, "matches.bin");
    const auto nmatch = rd<int32_t>(d, "nmatch.bin");
    const auto absperm = rd<int32_t>(d, "absperm.bin");
    const auto hapfull = rd<uint64_t>(d, "hapfull.bin");
    const auto typed = rd<int64_t>(d, "typed.bin");
    const auto af = rd<float>(d, "af.bin");
    std::vector<int32_t> segm(Mref);
    std::vector<uint8_t> common(Mref);
    std::vector<int2> sinfo(Mref);
    for (int m = 0; m < Mref; m++) {
        threadIdx.x = 0;
        blockIdx.x = (unsigned)m;
        blockDim.x = 1;
        eimp::segmap_kernel(typed.data(), M, Mref, af.data(), ntot, segm.data(), common.data(), sinfo.data());
    }
    const auto phased = rd<uint64_t>(d, "phased.bin");
    const auto gt = rd<uint8_t>(d, "gt.bin");
    const int ntiles = (nsites + 63) / 64, ldb = ntiles;
    const int nspans = (ntiles + eimp::DOS_SPAN - 1) / eimp::DOS_SPAN;
    std::vector<float> dos((size_t)nrows * nsites, -7.0f);
    std::vector<uint64_t> bits((size_t)nrows * ldb, 0x5A5A5A5A5A5A5A5Aull);
    for (long gw = 0; gw < (long)nhaps * nspans; gw++) {
        EmuWarp warp;
        std::vector<std::thread> lanes;
        for (int l = 0; l < 32; l++)
            lanes.emplace_back([&, l] {
                threadIdx.x = l;
                blockIdx.x = (unsigned)gw;
                blockDim.x = 32;
                emu_warp = &warp;
                (M < 131071 ? eimp::dosage_kernel<false, eimp::DOS_SPAN> : eimp::dosage_kernel<true, eimp::DOS_SPAN>)(
                    matches.data(), cap, nmatch.data(), absperm.data(), K, maps ? refmap.data() : nullptr,
                    hapfull.data(), wMref, sinfo.data(), phased.data(), wM, gt.data(), M, nhaps,
                    maps ? hapmap.data() : nullptr, mref_begin, nsites, impcalls,
                    dos.data(), nsites, bits.data(), ldb);
            });
        for (auto &x : lanes) x.join();
    }
    wr(d, "o_segm.bin", segm);
    wr(d, "o_sinfo.bin", sinfo);
    wr(d, "o_dos.bin", dos);
    wr(d, "o_bits.bin", bits);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
