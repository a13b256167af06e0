// Runs beam_kernel (generated host copy of eimp_b200/csrc/beam.cu) one
// target at a time under the warp emulator.
//
//   beam_emu <dir> [t0 t1]     one target per kernel call, each with a fresh arena
//   beam_emu <dir> queue       all targets through one call of one warp: the
//                              persistent loop takes them from the queue in
//                              longest-first order and reuses one arena
//
// <dir> holds the kernel inputs as raw little-endian arrays (params_i.bin,
// params_f.bin, gt.bin, monos.bin, splits.bin, nsplits.bin, calls.bin,
// ncalls.bin, cmd.bin, pbwt.bin, count0.bin, rowoff.bin, in the layout the
// device buffers have; optional startph.bin); the outputs are written next to
// them (o_*.bin).
// Each target gets its own arena and shared-memory block so the address
// sanitizer sees accesses past either.  Exit status 3: a divergent warp
// collective was seen.
#include "beam_emu.cpp"

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
    if (argc < 2) { fprintf(stderr, "usage: %s <dir> [t0 t1]\n", argv[0]); return 1; }
    const std::string d = argv[1];
    const bool queue = argc > 2 && std::string(argv[2]) == "queue";
    const auto pi = rd<int32_t>(d, "params_i.bin");
    const auto pf = rd<float>(d, "params_f.bin");
    const int ntgt = pi[0], M = pi[1];
    int t0 = argc > 2 && !queue ? atoi(argv[2]) : 0, t1 = argc > 3 ? atoi(argv[3]) : ntgt;
    if (t1 > ntgt) t1 = ntgt;
    eimp::BeamParams p;   // start phases: all Ref unless startph.bin is given
    p.K = pi[2]; p.H = pi[3]; p.P = pi[4]; p.Delta = pi[5]; p.Hf = pi[6]; p.Pf = pi[7]; p.Deltaf = pi[8];
    p.doPrePhasing = pi[9]; p.doRevPhasing = pi[10];
    p.expectIBDcM = pf[0]; p.pErr = pf[1]; p.pLimit = pf[2];
    p.minfixsize = pf[3]; p.maxfixsize = pf[4]; p.minfixthr = pf[5]; p.maxfixthr = pf[6];
    const auto gt = rd<uint8_t>(d, "gt.bin");
    const auto monos = rd<uint64_t>(d, "monos.bin");
    const auto splits = rd<int32_t>(d, "splits.bin");
    const auto nsplits = rd<int32_t>(d, "nsplits.bin");
    const auto calls = rd<int32_t>(d, "calls.bin");
    const auto ncalls = rd<int32_t>(d, "ncalls.bin");
    const auto cmd = rd<float>(d, "cmd.bin");
    const auto pbwt = rd<uint32_t>(d, "pbwt.bin");
    const auto count0 = rd<int32_t>(d, "count0.bin");
    const auto rowoff = rd<int64_t>(d, "rowoff.bin");
    // optional: start phases of the targets (0 = Ref)
    std::vector<uint8_t> startph;
    if (FILE *f = fopen((d + "/startph.bin").c_str(), "rb")) { fclose(f); startph = rd<uint8_t>(d, "startph.bin"); }
    const int wM = (int)eimp_W(M);
    const size_t kw = eimp_kw(p.K);
    const eimp::ArenaLayout al = eimp::arena_layout(p, M);
    const size_t smb = sizeof(eimp::WS) + eimp::beam_rows_bytes(p.K) + eimp::beam_canon_bytes(al.NH);
    std::vector<uint64_t> mats((size_t)ntgt * wM), pats((size_t)ntgt * wM);
    std::vector<float> dm((size_t)ntgt * M), dp((size_t)ntgt * M), tc(ntgt);
    std::vector<int32_t> nc(ntgt);
    std::vector<uint32_t> st(ntgt);
    if (queue) {
        std::vector<int32_t> order(ntgt, -1);
        threadIdx.x = 0;
        blockDim.x = 1;
        eimp::lpt_order_kernel(nsplits.data(), ntgt, order.data(), nullptr);
        for (int i = 1; i < ntgt; i++)   // longest first, ties by index
            if (nsplits[order[i - 1]] < nsplits[order[i]] ||
                (nsplits[order[i - 1]] == nsplits[order[i]] && order[i - 1] > order[i])) { fprintf(stderr, "order\n"); return 4; }
        uint8_t *arena = (uint8_t *)malloc(al.total);
        memset(arena, 0xA5, al.total);
        uint8_t *smem = (uint8_t *)aligned_alloc(16, (smb + 15) / 16 * 16);
        memset(smem, 0x5A, smb);
        int workq = 0;
        uint32_t status = 0;
        EmuWarp warp;
        std::vector<std::thread> lanes;
        for (int l = 0; l < 32; l++)
            lanes.emplace_back([&, l] {
                threadIdx.x = l;
                blockIdx.x = 0;
                blockDim.x = 32;
                emu_warp = &warp;
                emu_smem_ptr = smem;
                eimp::BeamParams pt = p;
                pt.startph = startph.empty() ? nullptr : startph.data();
                eimp::beam_kernel(pt, al, ntgt, M, gt.data(), monos.data(), splits.data(), nsplits.data(),
                                  calls.data(), ncalls.data(), cmd.data(), pbwt.data(), count0.data(), rowoff.data(),
                                  arena, al.total, mats.data(), pats.data(), dm.data(), dp.data(), tc.data(),
                                  nc.data(), &status, nullptr, order.data(), &workq);
            });
        for (auto &x : lanes) x.join();
        for (int t = 0; t < ntgt; t++) st[t] = status;
        free(arena);
        free(smem);
    }
    for (int t = t0; t < t1 && !queue; t++) {
        // fill patterns instead of zeros: the kernel must not read what it has not written
        uint8_t *arena = (uint8_t *)malloc(al.total);
        memset(arena, 0xA5, al.total);
        uint8_t *smem = (uint8_t *)aligned_alloc(16, (smb + 15) / 16 * 16);
        memset(smem, 0x5A, smb);
        const int64_t r0 = rowoff[t];
        const int64_t zero = 0;
        uint32_t status = 0;
        const int32_t first = 0;
        int workq = 0;
        EmuWarp warp;
        std::vector<std::thread> lanes;
        for (int l = 0; l < 32; l++)
            lanes.emplace_back([&, l] {
                threadIdx.x = l;
                blockIdx.x = 0;
                blockDim.x = 32;
                emu_warp = &warp;
                emu_smem_ptr = smem;
                eimp::BeamParams pt = p;
                pt.startph = startph.empty() ? nullptr : startph.data() + t;   // this target's entry at index 0
                eimp::beam_kernel(pt, al, 1, M, gt.data() + (size_t)t * M, monos.data() + (size_t)t * wM,
                                  splits.data() + (size_t)t * M, nsplits.data() + t, calls.data() + (size_t)t * M,
                                  ncalls.data() + t, cmd.data() + (size_t)t * (M + 1), pbwt.data() + 2 * r0 * kw,
                                  count0.data() + r0, &zero, arena, al.total, mats.data() + (size_t)t * wM,
                                  pats.data() + (size_t)t * wM, dm.data() + (size_t)t * M, dp.data() + (size_t)t * M,
                                  tc.data() + t, nc.data() + t, &status, nullptr, &first, &workq);
            });
        for (auto &x : lanes) x.join();
        st[t] = status;
        free(arena);
        free(smem);
    }
    wr(d, "o_mats.bin", mats); wr(d, "o_pats.bin", pats); wr(d, "o_dm.bin", dm); wr(d, "o_dp.bin", dp);
    wr(d, "o_tc.bin", tc); wr(d, "o_nc.bin", nc); wr(d, "o_st.bin", st);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
