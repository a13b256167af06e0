// Runs site_stats_kernel (generated host copy of
// eimp_b200/csrc/site_stats.cu) under the warp emulator, one block (all its
// warps, meeting at __syncthreads) at a time.
//
//   stats_emu <dir>
//
// <dir> holds the inputs as raw little-endian arrays in the layout of the
// device buffers: params_i.bin (ntgt, mref_begin, nsites, ldb, ldd, wM, ldp,
// M, Mref, overwriteCalls, improveCalls), params_f.bin (r2filter,
// maffilter), bits.bin, dos.bin, phased.bin, pdm.bin, pdp.bin, gt.bin,
// segm.bin, common.bin, af.bin, and haptgt.bin (one byte per target; empty:
// all diploid).  Outputs: o_ads.bin, o_gtbits.bin, o_ds.bin, o_gp.bin,
// o_site.bin (r2, af, maf as float, ac, an as int32, nsites each),
// o_pass.bin, o_conf.bin, o_icnt.bin and o_itot.bin (the --improveCalls
// counts and totals).  Exit status 3: a divergent warp collective.
#include "stats_emu.cpp"

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
    const auto pf = rd<float>(d, "params_f.bin");
    const auto bits = rd<uint64_t>(d, "bits.bin");
    const auto dos = rd<float>(d, "dos.bin");
    const auto phased = rd<uint64_t>(d, "phased.bin");
    const auto pdm = rd<float>(d, "pdm.bin");
    const auto pdp = rd<float>(d, "pdp.bin");
    const auto gt = rd<uint8_t>(d, "gt.bin");
    const auto segm = rd<int32_t>(d, "segm.bin");
    const auto common = rd<uint8_t>(d, "common.bin");
    const auto af = rd<float>(d, "af.bin");
    const auto haptgt = rd<uint8_t>(d, "haptgt.bin");
    eimp::SiteStatsArgs a;
    a.ntgt = pi[0]; a.mref_begin = pi[1]; a.nsites = pi[2]; a.ldb = pi[3]; a.ldd = pi[4]; a.wM = pi[5];
    a.ldp = pi[6]; a.M = pi[7]; a.overwriteCalls = pi[9]; a.improveCalls = pi[10];
    a.r2filter = pf[0]; a.maffilter = pf[1];
    a.bits = bits.data(); a.dos = dos.data(); a.phased = phased.data(); a.pdos_mat = pdm.data();
    a.pdos_pat = pdp.data(); a.gt = gt.data(); a.segm = segm.data(); a.common = common.data(); a.af = af.data();
    const size_t nh = 2 * (size_t)a.ntgt, ns = a.nsites;
    // outputs sized exactly (the address sanitizer sees any access past them)
    std::vector<float> ads(nh * ns, -7.0f), ds((size_t)a.ntgt * ns), gp(3 * (size_t)a.ntgt * ns);
    std::vector<uint64_t> gtbits(nh * a.ldb, 0);
    std::vector<float> site_f(3 * ns);
    std::vector<int32_t> site_i(2 * ns);
    std::vector<uint8_t> pass(ns);
    std::vector<unsigned long long> conf(1, 0), icnt(5, 0);
    std::vector<double> itot(5, 0.0);
    a.haptgt = haptgt.empty() ? nullptr : haptgt.data();
    a.icnt = icnt.data();
    a.itot = itot.data();
    a.ads = ads.data(); a.lda = (int)ns; a.gtbits = gtbits.data(); a.ldg = a.ldb; a.ds = ds.data(); a.gp = gp.data();
    a.r2 = site_f.data(); a.af_out = site_f.data() + ns; a.maf = site_f.data() + 2 * ns;
    a.ac = site_i.data(); a.an = site_i.data() + ns; a.pass = pass.data(); a.conflicts = conf.data();
    // whole blocks: the producer warps and the summing warp meet at __syncthreads
    const int blocks = (a.nsites + 31) / 32, nw = eimp::SS_PROD + 1;
    for (int b = 0; b < blocks; b++) {
        std::vector<EmuWarp> warps(nw);
        EmuBarrier block;
        block.n = 32 * nw;
        std::vector<std::thread> threads;
        for (int t = 0; t < 32 * nw; t++)
            threads.emplace_back([&, t] {
                threadIdx.x = t;
                blockIdx.x = b;
                blockDim.x = 32 * nw;
                emu_warp = &warps[t / 32];
                emu_block = &block;
                if (a.haptgt) eimp::site_stats_kernel<true, true, true>(a);
                else eimp::site_stats_kernel<true, true, false>(a);
            });
        for (auto &x : threads) x.join();
    }
    wr(d, "o_ads.bin", ads); wr(d, "o_gtbits.bin", gtbits); wr(d, "o_ds.bin", ds); wr(d, "o_gp.bin", gp);
    wr(d, "o_site_f.bin", site_f); wr(d, "o_site_i.bin", site_i); wr(d, "o_pass.bin", pass);
    wr(d, "o_conf.bin", conf);
    wr(d, "o_icnt.bin", icnt);
    wr(d, "o_itot.bin", itot);
    if (emu_divergence.load()) { fprintf(stderr, "divergent warp collectives: %d\n", emu_divergence.load()); return 3; }
    return 0;
}
