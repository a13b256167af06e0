// Runs the condensed-reference kernel (generated host copy of
// eimp_b200/csrc/phase_prep.cu: cref_kernel) under the warp emulator, whole
// blocks one after the other.
//
//   cref_emu <dir>
//
// <dir> holds params_i.bin (ntgt, M, nhaps, K), gt.bin (ntgt x M uint8),
// hapmajor.bin (nhaps x W(M) words), besthaps.bin (ntgt x K int32),
// splits.bin (ntgt x M int32), nsplits.bin (ntgt int32) and rowoff.bin
// (ntgt+1 int64).  Output: o_cref.bin (rows x W(K) words).  Exit status 3: a
// divergent warp collective.
#include "cref_emu.cpp"

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
    const auto gt = rd<uint8_t>(d, "gt.bin");
    const auto hapmajor = rd<uint64_t>(d, "hapmajor.bin");
    const auto besthaps = rd<int32_t>(d, "besthaps.bin");
    const auto splits = rd<int32_t>(d, "splits.bin");
    const auto nsplits = rd<int32_t>(d, "nsplits.bin");
    const auto rowoff = rd<int64_t>(d, "rowoff.bin");
    const int ntgt = pi[0], M = pi[1], nhaps = pi[2], K = pi[3];
    const int wM = (int)eimp_W(M), wK = (int)eimp_W(K);
    std::vector<uint64_t> cref((size_t)rowoff[ntgt] * wK, 0xdeadbeefdeadbeefull);
    const int nthreads = 32 * eimp::CREF_WARPS, nwarps = eimp::CREF_WARPS;
    const int gy = (2 * wK + eimp::CREF_WARPS - 1) / eimp::CREF_WARPS;
    for (int bx = 0; bx < ntgt; bx++)
        for (int by = 0; by < gy; by++) {
            std::vector<uint64_t> smem((size_t)3 * wM, 0x5a5a5a5a5a5a5a5aull);   // exact size: ASan sees overruns
            std::vector<EmuWarp> warps(nwarps);
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
                    eimp::cref_kernel(gt.data(), M, hapmajor.data(), wM, nhaps, besthaps.data(), K, splits.data(),
                                      nsplits.data(), rowoff.data(), cref.data(), nullptr);
                });
            for (auto &x : threads) x.join();
        }
    wr(d, "o_cref.bin", cref);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
