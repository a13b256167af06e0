// Runs the reference PBWT's checkpoint and fill kernels (generated host copy
// of eimp_b200/csrc/imp_kernels.cu: refpbwt_ckpt_kernel, refpbwt_fill_kernel)
// under the warp emulator, whole 1024-thread blocks one after the other.
//
//   refpbwt_emu <dir>
//
// <dir> holds params_i.bin (M, K, wN, orders_in_smem, stage_rows) and
// sitemajor.bin (M x wN words).  Outputs: o_compr.bin (M x 2*ceil(K/32)
// uint32), o_absperm.bin ((M+1) x K int32), o_count0.bin (M int32).  The
// orders live in the block's shared memory or in a global scratch buffer as
// the flags say (the launcher picks by the shared-memory size), with one
// round of loads in flight in shared memory and eight in global memory, as
// the launcher runs them.  Exit status
// 3: a divergent warp collective.
#include "refpbwt_emu.cpp"

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

template <class F> static void run_blocks(int nblocks, int nthreads, size_t smem_bytes, F kern) {
    for (int b = 0; b < nblocks; b++) {
        std::vector<uint64_t> smem((smem_bytes + 7) / 8, 0x5a5a5a5a5a5a5a5aull);   // exact size: ASan sees overruns
        std::vector<EmuWarp> warps(nthreads / 32);
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
                kern();
            });
        for (auto &x : threads) x.join();
    }
}

int main(int argc, char **argv) {
    if (argc < 2) { fprintf(stderr, "usage: %s <dir>\n", argv[0]); return 1; }
    const std::string d = argv[1];
    const auto pi = rd<int32_t>(d, "params_i.bin");
    const int M = pi[0], K = pi[1], wN = pi[2], in_smem = pi[3], stage = pi[4];
    const auto sm = rd<uint64_t>(d, "sitemajor.bin");
    const int nwords = (K + 31) / 32;
    std::vector<uint32_t> compr((size_t)M * 2 * nwords, 0xdeadbeefu);
    std::vector<int32_t> absperm((size_t)(M + 1) * K, -1), count0(M, -1);
    std::vector<int32_t> scratch(in_smem ? 0 : ((size_t)K * 9 + 3) / 4);
    const size_t ck_smem = (size_t)(1024 + 32) * 4 + (stage ? (size_t)eimp::RP_BITS * wN * 8 : 0) +
                           (in_smem ? (size_t)K * 9 : 0);
    run_blocks(1, 1024, ck_smem, [&] {
        if (in_smem) eimp::refpbwt_ckpt_kernel<1>(sm.data(), M, K, wN, absperm.data(), nullptr, stage);
        else eimp::refpbwt_ckpt_kernel<8>(sm.data(), M, K, wN, absperm.data(), scratch.data(), stage);
    });
    const size_t fill_smem = (size_t)2 * wN * 4 + (size_t)nwords * 4 + (size_t)(nwords + 1) * 4 + 33 * 4;
    run_blocks((M + eimp::RP_CK - 1) / eimp::RP_CK, 1024, fill_smem, [&] {
        eimp::refpbwt_fill_kernel(sm.data(), M, K, wN, compr.data(), absperm.data(), count0.data());
    });
    wr(d, "o_compr.bin", compr); wr(d, "o_absperm.bin", absperm); wr(d, "o_count0.bin", count0);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
