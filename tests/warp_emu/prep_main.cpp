// Runs the phasing preparation kernels (generated host copy of
// eimp_b200/csrc/phase_prep.cu: hamming_kernel, besthaps_kernel,
// monos_calls_kernel) under the warp emulator, whole blocks one after the
// other, in the order the library launches them.
//
//   prep_emu <dir>
//
// <dir> holds params_i.bin (ntgt, M, nhaps, K, tb[, self0, use_haploid]),
// haploid.bin (nhaps / 2 uint8, when use_haploid), params_f.bin
// (cMmaxsplit), gt.bin (ntgt x M uint8), hapmajor.bin (nhaps x W(M) words)
// and cm.bin (M float).  Outputs: o_nerr.bin (ntgt x nhaps uint32),
// o_besthaps.bin (ntgt x K int32), o_flags.bin (ntgt x W(nhaps) words),
// o_monos.bin (ntgt x W(M) words),
// o_splits.bin / o_calls.bin (ntgt x M int32), o_cmdiffs.bin (ntgt x (M+1)
// float), o_nsplits.bin / o_ncalls.bin (ntgt int32).  Exit status 3: a
// divergent warp collective.
#include "prep_emu.cpp"

#include <functional>
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

// one block of nthreads threads with smem_bytes of dynamic shared memory
static void run_block(unsigned bx, unsigned by, int nthreads, size_t smem_bytes, const std::function<void()> &body) {
    std::vector<uint64_t> smem((smem_bytes + 7) / 8 + 1, 0x5a5a5a5a5a5a5a5aull);
    std::vector<EmuWarp> warps((nthreads + 31) / 32);
    EmuBarrier block;
    block.n = nthreads;
    std::vector<std::thread> threads;
    for (int t = 0; t < nthreads; t++)
        threads.emplace_back([&, t] {
            threadIdx.x = t;
            blockIdx.x = bx;
            blockIdx.y = by;
            blockDim.x = nthreads;
            emu_warp = &warps[t / 32];
            emu_block = &block;
            emu_smem_ptr = reinterpret_cast<uint8_t *>(smem.data());
            body();
        });
    for (auto &x : threads) x.join();
}

int main(int argc, char **argv) {
    if (argc < 2) { fprintf(stderr, "usage: %s <dir>\n", argv[0]); return 1; }
    const std::string d = argv[1];
    const auto pi = rd<int32_t>(d, "params_i.bin");
    const auto pf = rd<float>(d, "params_f.bin");
    const auto gt = rd<uint8_t>(d, "gt.bin");
    const auto hapmajor = rd<uint64_t>(d, "hapmajor.bin");
    const auto cm = rd<float>(d, "cm.bin");
    const int ntgt = pi[0], M = pi[1], nhaps = pi[2], K = pi[3], tb = pi[4];
    const int self0 = pi.size() > 5 ? pi[5] : -1;
    const std::vector<uint8_t> hapl = pi.size() > 6 && pi[6] ? rd<uint8_t>(d, "haploid.bin") : std::vector<uint8_t>();
    const uint8_t *haploid = hapl.empty() ? nullptr : hapl.data();
    const float cMmaxsplit = pf[0];
    const int wM = (int)eimp_W(M), wN = (int)eimp_W(nhaps);
    std::vector<uint32_t> nerr((size_t)ntgt * nhaps, 0xdeadbeefu);
    std::vector<int32_t> besthaps((size_t)ntgt * K, -7);
    std::vector<uint64_t> flags((size_t)ntgt * wN, 0), monos((size_t)ntgt * wM, 0);
    std::vector<int32_t> splits((size_t)ntgt * M, -7), calls((size_t)ntgt * M, -7), nsplits(ntgt, -7), ncalls(ntgt, -7);
    std::vector<float> cmdiffs((size_t)ntgt * (M + 1), -7.0f);

    const unsigned gx = (unsigned)((ntgt + tb - 1) / tb);
    const unsigned gy = (unsigned)((nhaps + eimp::HAM_WARPS * eimp::HAM_HPW - 1) / (eimp::HAM_WARPS * eimp::HAM_HPW));
    const size_t hsm = (size_t)2 * wM * 8 * tb;
    for (unsigned bx = 0; bx < gx; bx++)
        for (unsigned by = 0; by < gy; by++)
            run_block(bx, by, 32 * eimp::HAM_WARPS, hsm, [&] {
                if (tb == 8) eimp::hamming_kernel<8>(gt.data(), ntgt, M, hapmajor.data(), nhaps, wM, nerr.data(), self0, haploid);
                else if (tb == 4) eimp::hamming_kernel<4>(gt.data(), ntgt, M, hapmajor.data(), nhaps, wM, nerr.data(), self0, haploid);
                else if (tb == 2) eimp::hamming_kernel<2>(gt.data(), ntgt, M, hapmajor.data(), nhaps, wM, nerr.data(), self0, haploid);
                else eimp::hamming_kernel<1>(gt.data(), ntgt, M, hapmajor.data(), nhaps, wM, nerr.data(), self0, haploid);
            });
    wr(d, "o_nerr.bin", nerr);
    for (int t = 0; t < ntgt; t++)
        run_block(t, 0, 512, 0, [&] {
            eimp::besthaps_kernel(gt.data(), M, hapmajor.data(), nhaps, wM, K, nerr.data(), besthaps.data(),
                                  flags.data(), wN, self0, haploid);
        });
    for (int t = 0; t < ntgt; t++)
        run_block(t, 0, 256, (size_t)2 * wM * 8, [&] {
            eimp::monos_calls_kernel(gt.data(), M, hapmajor.data(), wM, besthaps.data(), K, cm.data(), cMmaxsplit,
                                     monos.data(), splits.data(), calls.data(), cmdiffs.data(), nsplits.data(),
                                     ncalls.data(), nullptr);
        });
    wr(d, "o_besthaps.bin", besthaps);
    wr(d, "o_flags.bin", flags);
    wr(d, "o_monos.bin", monos);
    wr(d, "o_splits.bin", splits);
    wr(d, "o_calls.bin", calls);
    wr(d, "o_cmdiffs.bin", cmdiffs);
    wr(d, "o_nsplits.bin", nsplits);
    wr(d, "o_ncalls.bin", ncalls);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
