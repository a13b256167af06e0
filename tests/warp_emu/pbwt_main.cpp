// Runs the condensed-reference PBWT kernel (generated host copy of
// eimp_b200/csrc/phase_prep.cu: pbwt_kernel) under the warp emulator, whole
// blocks one after the other.
//
//   pbwt_emu <dir>
//
// <dir> holds params_i.bin (ntgt, K, rowstride, emit_padded, wpt),
// rowoff.bin (ntgt+1 int64) and cref.bin (rows x W(K) words).  Outputs:
// o_pbwt.bin (2 * rows x rowstride uint32, forward then backward rows of each
// target), o_count0.bin (rows int32).  Exit status 3: a divergent warp
// collective.
#include "pbwt_emu.cpp"

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
    const auto rowoff = rd<int64_t>(d, "rowoff.bin");
    const auto cref = rd<uint64_t>(d, "cref.bin");
    const int ntgt = pi[0], K = pi[1], rowstride = pi[2], emit_padded = pi[3], wpt = pi[4];
    const size_t rows = (size_t)rowoff[ntgt];
    std::vector<uint32_t> pbwt(2 * rows * rowstride, 0xdeadbeefu);
    std::vector<int32_t> count0(rows, -7);
    const int nwords = (K + 31) / 32, nthreads = ((nwords + wpt - 1) / wpt + 31) / 32 * 32, nwarps = nthreads / 32;
    const size_t smem_bytes = eimp::pbwt_smem(K);
    for (int b = 0; b < 2 * ntgt; b++) {
        std::vector<uint64_t> smem((smem_bytes + 7) / 8, 0x5a5a5a5a5a5a5a5aull);   // exact size: ASan sees overruns
        std::vector<EmuWarp> warps(nwarps);
        EmuBarrier block;
        block.n = nthreads;
        std::vector<std::thread> threads;
        for (int t = 0; t < nthreads; t++)
            threads.emplace_back([&, t] {
                threadIdx.x = t;
                blockIdx.x = b;
                blockDim.x = nthreads;
                emu_warp = &warps[t / 32];
                emu_block = &block;
                emu_smem_ptr = reinterpret_cast<uint8_t *>(smem.data());
                if (wpt == 1)
                    eimp::pbwt_kernel<1>(cref.data(), rowoff.data(), K, pbwt.data(), rowstride, emit_padded,
                                          count0.data(), nullptr);
                else
                    eimp::pbwt_kernel<2>(cref.data(), rowoff.data(), K, pbwt.data(), rowstride, emit_padded,
                                          count0.data(), nullptr);
            });
        for (auto &x : threads) x.join();
    }
    wr(d, "o_pbwt.bin", pbwt);
    wr(d, "o_count0.bin", count0);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
