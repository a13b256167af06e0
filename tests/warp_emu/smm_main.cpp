// Runs the set-maximal match kernels (generated host copy of the match
// section of eimp_b200/csrc/imp_kernels.cu) one target haplotype at a time
// under the warp emulator.
//
//   smm_emu <dir> <kernel> [pool]   kernel 0: smm_kernel, 1: smm_compact_kernel
//                                   (32-bit intervals), 2: smm_compact_kernel (16-bit
//                                   intervals); pool: global tree pools of the
//                                   compact kernels' first pass (slots, default 0)
//
// Both launches of launch_smm run: the small node pool first, then the retry
// pass with the large pool.  <dir> holds the inputs as raw little-endian arrays in the layout of the
// device buffers: params_i.bin (nhaps, M, K, setmaxerrors, cap[, nrows, use_hapmap]), compr.bin
// (M x kw u32), count0.bin (M i32), phased.bin (nhaps x W(M) u64), gt.bin
// (nhaps/2 x M u8).  Outputs: o_matches.bin (nhaps x cap int4), o_nmatch.bin,
// o_status.bin, o_retried.bin (haplotypes redone by the retry pass).  With use_hapmap,
// the phased rows and outputs have nrows rows (the target haplotypes) and
// hapmap.bin lists the nhaps of them that are searched.  Each haplotype gets its own shared-memory block so the
// address sanitizer sees accesses past it.  Exit status 3: a divergent warp
// collective was seen.
#include "smm_emu.cpp"

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
    if (argc < 3) { fprintf(stderr, "usage: %s <dir> <kernel>\n", argv[0]); return 1; }
    const std::string d = argv[1];
    const int which = atoi(argv[2]);
    const int pool_slots = argc > 3 ? atoi(argv[3]) : 0;
    const auto pi = rd<int32_t>(d, "params_i.bin");
    const int nhaps = pi[0], M = pi[1], K = pi[2], sme = pi[3], cap = pi[4];
    const int nrows = pi.size() > 5 ? pi[5] : nhaps;
    const std::vector<int32_t> hapmap = pi.size() > 6 && pi[6] ? rd<int32_t>(d, "hapmap.bin") : std::vector<int32_t>();
    const int32_t *hm = hapmap.empty() ? nullptr : hapmap.data();
    const auto compr = rd<uint32_t>(d, "compr.bin");
    const auto count0 = rd<int32_t>(d, "count0.bin");
    const auto phased = rd<uint64_t>(d, "phased.bin");
    const auto gt = rd<uint8_t>(d, "gt.bin");
    const int wM = (int)eimp_W(M);
    std::vector<int4> matches((size_t)nrows * cap, int4{-7, -7, -7, -7});
    std::vector<int32_t> nmatch(nrows, -7);
    uint32_t status = 0;
    int retried = 0;
    // global tree pools of the first pass (exact size: the address sanitizer
    // sees any access past the slots handed out) and their counter
    const size_t slot_bytes = which == 2 ? sizeof(eimp::SmmWarpSmemC<SMM_NODES_RETRY, uint16_t>)
                                         : sizeof(eimp::SmmWarpSmemC<SMM_NODES_RETRY, int>);
    std::vector<uint64_t> gpool(pool_slots ? (pool_slots * slot_bytes + 7) / 8 : 0, 0x5a5a5a5a5a5a5a5aull);
    int gnext = 0;
    void *gp = pool_slots ? (void *)gpool.data() : nullptr;
    // the launches of launch_smm: the small node pool, then the retry pass
    for (int pass = 0; pass < 2; pass++) {
        const size_t smb = which == 2 ? (pass ? sizeof(eimp::SmmWarpSmemC<SMM_NODES_RETRY, uint16_t>)
                                              : sizeof(eimp::SmmWarpSmemC<SMM_NODES, uint16_t>))
                           : which ? (pass ? sizeof(eimp::SmmWarpSmemC<SMM_NODES_RETRY>)
                                           : sizeof(eimp::SmmWarpSmemC<SMM_NODES>))
                                   : (pass ? sizeof(eimp::SmmWarpSmem<SMM_NODES_RETRY>)
                                           : sizeof(eimp::SmmWarpSmem<SMM_NODES>));
        for (int h = 0; h < nhaps; h++) {
            if (pass) retried += nmatch[hm ? hm[h] : h] == eimp::SMM_RETRY;
            // a fill pattern instead of zeros: the kernel must not read what it has not written
            uint8_t *smem = (uint8_t *)aligned_alloc(16, (smb + 15) / 16 * 16);
            memset(smem, 0x5A, smb);
            EmuWarp warp;
            std::vector<std::thread> lanes;
            for (int l = 0; l < 32; l++)
                lanes.emplace_back([&, l] {
                    threadIdx.x = l;
                    blockIdx.x = h;
                    emu_warp = &warp;
                    emu_smem_ptr = smem;
                    using Big16 = eimp::SmmWarpSmemC<SMM_NODES_RETRY, uint16_t>;
                    using Big32 = eimp::SmmWarpSmemC<SMM_NODES_RETRY, int>;
                    if (which == 2) {
                        auto kern = pass ? eimp::smm_compact_kernel<SMM_NODES_RETRY, 1, true, uint16_t>
                                         : eimp::smm_compact_kernel<SMM_NODES, 1, false, uint16_t>;
                        kern(compr.data(), count0.data(), M, K, phased.data(), wM, gt.data(), nhaps, hm, sme,
                             matches.data(), cap, nmatch.data(), &status, pass ? nullptr : (Big16 *)gp,
                             pass ? 0 : pool_slots, pass ? nullptr : &gnext);
                    } else if (which == 1) {
                        auto kern = pass ? eimp::smm_compact_kernel<SMM_NODES_RETRY, 1, true, int>
                                         : eimp::smm_compact_kernel<SMM_NODES, 1, false, int>;
                        kern(compr.data(), count0.data(), M, K, phased.data(), wM, gt.data(), nhaps, hm, sme,
                             matches.data(), cap, nmatch.data(), &status, pass ? nullptr : (Big32 *)gp,
                             pass ? 0 : pool_slots, pass ? nullptr : &gnext);
                    } else {
                        auto kern = pass ? eimp::smm_kernel<SMM_NODES_RETRY, 1, true> : eimp::smm_kernel<SMM_NODES, 1, false>;
                        kern(compr.data(), count0.data(), M, K, phased.data(), wM, gt.data(), nhaps, hm, sme,
                             matches.data(), cap, nmatch.data(), &status);
                    }
                });
            for (auto &x : lanes) x.join();
            free(smem);
        }
    }
    wr(d, "o_retried.bin", std::vector<int32_t>{retried, gnext});
    wr(d, "o_matches.bin", matches);
    wr(d, "o_nmatch.bin", nmatch);
    wr(d, "o_status.bin", std::vector<uint32_t>{status});
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
